// TMA-staged variant of the fused step: the populations a block needs for one level are brought into shared memory
// by tensor-memory-accelerator box copies, several levels ahead of the level being computed, so the HBM latency is
// hidden by the copy engine instead of by registers and warps.
//
// Block = 32 x TY columns walking its z-slab level by level. For level k and population q the pull sources of the
// block's cells form one box of the population plane: rows j0 - cy .. j0 - cy + TY - 1, level k - cz, x from x0 - cx.
// TMA x starts must be 16-byte aligned, so directions with cx != 0 use a "wide" box that starts H elements early
// (H = 16 bytes / element size) and is 32 + 2H wide; cx = 0 uses a 32-wide box at x0. Out-of-range rows, levels and
// columns are zero-filled by the copy engine; only cells that take the interior path (every source fluid and inside
// the domain) read from these boxes, the others use the global-memory stream of fused.cuh.
//
// One thread issues the 26 box copies of a level into a stage and arms the stage's mbarrier with the byte count;
// every thread waits on the barrier with a bound (the global timer): a wait that runs out sets the error word
// D.err, the block stops computing, and thread 0 waits (again bounded) for the copies it issued before the block
// exits. No multicast: each block copies its own boxes from this GPU's memory.
#pragma once

#include <cuda.h>

#include "fused.cuh"

namespace ahx {

struct TmaMaps {
  CUtensorMap fw, fn, gw, gn;   // f / g state being read: wide (cx != 0) and narrow (cx = 0) boxes
};

template <class S>
struct TmaGeom {
  static constexpr int H = 16 / (int)sizeof(S);          // x halo of a wide box, one 16-byte granule
  static constexpr int WW = 32 + 2 * H;                   // wide box width
  template <int TY>
  static constexpr int wide_bytes() { return WW * TY * (int)sizeof(S); }
  template <int TY>
  static constexpr int narrow_bytes() { return 32 * TY * (int)sizeof(S); }
  // byte offset of population q's box (f: q < 19, g: 19 + q) inside a stage; boxes stay 128-byte aligned
  template <int TY>
  static constexpr int box_offset(int slot) {
    int off = 0;
    for (int s = 0; s < slot; ++s) {
      const int cx = s < 19 ? kC19[s][0] : kC7[s - 19][0];
      off += cx != 0 ? wide_bytes<TY>() : narrow_bytes<TY>();
    }
    return off;
  }
  template <int TY>
  static constexpr int stage_bytes() { return box_offset<TY>(26); }
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ uint64_t global_timer_ns() {
  uint64_t t;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
  return t;
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arm(uint64_t* bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t* bar, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}

// wait for a stage with a time bound; false when the bound ran out
__device__ __forceinline__ bool mbar_wait_bounded(uint64_t* bar, unsigned parity, uint64_t limit_ns) {
  if (mbar_try_wait(bar, parity)) return true;
  const uint64_t t0 = global_timer_ns();
  while (!mbar_try_wait(bar, parity)) {
    if (global_timer_ns() - t0 > limit_ns) return false;
  }
  return true;
}

// One box copy. The tensor map (64 B), destination (128 B) and barrier (8 B) alignments the copy engine requires are
// checked first: a violation sets the error word and skips the copy (its stage then never completes and the block
// aborts through its bounded wait) instead of faulting.
__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int x, int y, int z, int w,
                                            uint64_t* bar, int* err) {
  if (((reinterpret_cast<uint64_t>(map) & 63) | (smem_u32(dst) & 127) | (smem_u32(bar) & 7)) != 0) {
    atomicExch(err, 2);
    return;
  }
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], "
      "[%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(w), "r"(smem_u32(bar))
      : "memory");
}

constexpr uint64_t kStageWaitLimitNs = 200ull * 1000 * 1000;   // 200 ms: far beyond any real copy

template <class S, int TY>
__device__ __forceinline__ void tma_issue_level(const TmaMaps& M, unsigned char* stage, uint64_t* bar, int x0,
                                                int j0, int k, int* err) {
  using G = TmaGeom<S>;
  mbar_arm(bar, (unsigned)G::template stage_bytes<TY>());
  static_for<19>([&](auto Q) {
    constexpr int q = Q;
    constexpr int cx = kC19[q][0], cy = kC19[q][1], cz = kC19[q][2];
    constexpr int off = G::template box_offset<TY>(q);
    if constexpr (cx != 0) tma_load_4d(stage + off, &M.fw, x0 - G::H, j0 - cy, k - cz, q, bar, err);
    else tma_load_4d(stage + off, &M.fn, x0, j0 - cy, k - cz, q, bar, err);
  });
  static_for<7>([&](auto Q) {
    constexpr int q = Q;
    constexpr int cx = kC7[q][0], cy = kC7[q][1], cz = kC7[q][2];
    constexpr int off = G::template box_offset<TY>(19 + q);
    if constexpr (cx != 0) tma_load_4d(stage + off, &M.gw, x0 - G::H, j0 - cy, k - cz, q, bar, err);
    else tma_load_4d(stage + off, &M.gn, x0, j0 - cy, k - cz, q, bar, err);
  });
}

// populations of an interior cell from the staged boxes (the same values stream_interior loads)
template <class S, int TY>
__device__ __forceinline__ void stage_read(const unsigned char* stage, int tx, int ty,
                                           Cell<typename Codec<S>::Real>& X) {
  using R = typename Codec<S>::Real;
  using K = Codec<S>;
  using G = TmaGeom<S>;
  static_for<19>([&](auto Q) {
    constexpr int q = Q;
    constexpr int cx = kC19[q][0];
    constexpr int off = G::template box_offset<TY>(q);
    const S* box = reinterpret_cast<const S*>(stage + off);
    const S v = cx != 0 ? box[ty * G::WW + tx + G::H - cx] : box[ty * 32 + tx];
    X.f[q] = K::dec_f(v, R(w19(q)));
  });
  static_for<7>([&](auto Q) {
    constexpr int q = Q;
    constexpr int cx = kC7[q][0];
    constexpr int off = G::template box_offset<TY>(19 + q);
    const S* box = reinterpret_cast<const S*>(stage + off);
    const S v = cx != 0 ? box[ty * G::WW + tx + G::H - cx] : box[ty * 32 + tx];
    X.g[q] = K::dec_g(v);
  });
}

// dynamic shared memory of the staged step: 128 bytes of alignment slack, DEPTH stages (each a multiple of 128 bytes),
// a 128-byte slot for the DEPTH barriers, then the nz-entry float4 profile (so it stays 16-byte aligned)
constexpr int kBarSlot = 128;
template <class S, int TY, int DEPTH>
constexpr size_t tma_smem_bytes(int nz) {
  static_assert(8 * DEPTH <= kBarSlot, "barriers fit their slot");
  static_assert(TmaGeom<S>::template stage_bytes<TY>() % 128 == 0, "stages keep 128-byte alignment");
  return 128 + (size_t)DEPTH * TmaGeom<S>::template stage_bytes<TY>() + kBarSlot + 16 * (size_t)nz;
}

template <class S, bool FAST, int TY, int DEPTH>
__device__ __forceinline__ void step_tma_block(const DomainView& D, const TmaMaps& M, int zslab) {
  static_assert(!kDitherOf<S>, "the staged kernel takes no dither (stochastic-rounding storages use the plain kernel)");
  static_assert(!kLevelPairs<StoreF<S>>, "the staged kernel's boxes are single levels (level-paired planes use the plain "
                                         "kernel)");
  using R = typename Codec<S>::Real;
  using G = TmaGeom<S>;
  constexpr int STAGE = G::template stage_bytes<TY>();
  extern __shared__ unsigned char tma_smem_raw[];
  __shared__ ParamsHead sP;
  __shared__ int s_kmin;
  __shared__ int s_abort;
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(tma_smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + (size_t)DEPTH * STAGE);
  float4* prof = reinterpret_cast<float4*>(base + (size_t)DEPTH * STAGE + kBarSlot);

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * 32 + tx;
  const int x0 = blockIdx.x * 32, j0 = blockIdx.y * TY;
  const int k0 = blockIdx.z * zslab;
  const int k1 = min(D.nz, k0 + zslab);
  if (tid < 16) reinterpret_cast<int*>(&sP)[tid] = reinterpret_cast<const int*>(D.params)[tid];
  const float4* gprof = reinterpret_cast<const float4*>(D.params + 64);
  for (int z = tid; z < D.nz; z += 32 * TY) prof[z] = gprof[z];
  if (tid == 0) {
    s_kmin = k1;
    s_abort = 0;
    for (int s = 0; s < DEPTH; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const ParamsHead& P = sP;
  const RelaxConst RK = relax_const(P);
  const int i = x0 + tx, j = j0 + ty;
  const bool active = i < D.nx && j < D.ny;
  Column<R> C;
  if (active) {
    load_column(D, P, i, j, C);
    atomicMin(&s_kmin, max(k0, C.kg));
  }
  __syncthreads();
  const int kb = s_kmin;   // first level with a fluid cell in this block's slab
  if (tid == 0)
    for (int d = 0; d < DEPTH && kb + d < k1; ++d)
      tma_issue_level<S, TY>(M, base + (size_t)d * STAGE, &bars[d], x0, j0, kb + d, D.err);
  const uint32_t cbase = (uint32_t)j * (uint32_t)D.px + (uint32_t)i;
  int it = 0;
  for (int k = kb; k < k1; ++k, ++it) {
    const int s = it % DEPTH;
    const unsigned parity = (unsigned)((it / DEPTH) & 1);
    unsigned char* stage = base + (size_t)s * STAGE;
    // a set error word (from this or another block) stops the step early instead of waiting on stages
    if (*reinterpret_cast<volatile int*>(D.err) != 0) s_abort = 1;
    else if (!mbar_wait_bounded(&bars[s], parity, kStageWaitLimitNs)) s_abort = 1;
    if (active && k >= C.kg && !s_abort) {
      const uint32_t n = (uint32_t)k * D.ps + cbase;
      Cell<R> X;
      if (!C.face && k >= C.kint && k < D.nz - 1) {
        int zagl = k - C.ktc;
        if (zagl < 0) zagl = 0;
        if (zagl > D.nz - 1) zagl = D.nz - 1;
        const float4 pr = prof[zagl];
        X.uI = R(pr.x);
        X.vI = R(pr.y);
        X.kb = R(pr.z);
        stage_read<S, TY>(stage, tx, ty, X);
      } else {
        stream_cell<S>(D, P, prof, C, k, cbase, X);
      }
      Macro<R> Mc;
      if constexpr (FAST) {
        fast_update<S>(D, P, RK, C, k, n, n, X, Mc, 0u);
      } else {
        moments_forces<R>(P, C, k, D.nz, X, Mc);
        collide_store<S>(D, P, C, k, n, n, X, Mc, 0u);
      }
    }
    __syncthreads();   // stage s consumed by every thread
    if (s_abort) {
      if (tid == 0) {
        atomicExch(D.err, 1);
        // wait (bounded) for the copies still in flight into this block's stages before it exits
        for (int L = k; L < min(k1, k + DEPTH); ++L) {
          const int iL = L - kb;
          mbar_wait_bounded(&bars[iL % DEPTH], (unsigned)((iL / DEPTH) & 1), kStageWaitLimitNs);
        }
      }
      break;
    }
    if (tid == 0 && k + DEPTH < k1) tma_issue_level<S, TY>(M, stage, &bars[s], x0, j0, k + DEPTH, D.err);
  }
  if (tid == 0 && !s_abort) {
    // before the block exits, every stage it armed must have completed its last phase (bounded wait)
    for (int st = 0; st < DEPTH; ++st) {
      const int uses = (k1 - kb > st) ? ((k1 - kb - st + DEPTH - 1) / DEPTH) : 0;
      if (uses > 0 && !mbar_wait_bounded(&bars[st], (unsigned)((uses - 1) & 1), kStageWaitLimitNs))
        atomicExch(D.err, 1);
    }
  }
}

}  // namespace ahx

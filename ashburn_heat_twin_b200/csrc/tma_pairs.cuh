// TMA-staged paired step of the 16-bit storages: the pull sources of a block's interior cell pairs are brought into
// shared memory by tensor-memory-accelerator box copies a few level pairs ahead, so the warps issue only shared-memory
// reads with immediate offsets (no per-population address arithmetic) and never wait on HBM themselves.
//
// Layout read: a 16-bit storage keeps the levels (2t, 2t + 1) of a population plane in one 32-bit word (lvl in
// lattice.cuh), so the plane is a [pair][row][x] array of words. The cell pair (2t, 2t + 1) of population q pulls the
// levels (2t - cz, 2t + 1 - cz) of its source column: for cz = 0 word t; for cz = +1 the high half of word t - 1 and
// the low half of word t; for cz = -1 the high half of word t and the low half of word t + 1. Stage t holds, for every
// population slot (19 f, 7 g), the box of words the block's 32 x TY columns pull from, at pair t for cz >= 0 and at
// pair t + 1 for cz = -1: rows y0 - cy .. y0 - cy + TY - 1, words x0 - cx ..; directions with cx != 0 take a box 4
// words (16 bytes) wider on each side, so every box starts on a 16-byte boundary (x0 is 16 + 32 bx words). A thread
// keeps the word it read from each cz != 0 box in a register for its next pair (word t of cz = +1 is the next pair's
// word t - 1; word t + 1 of cz = -1 is its word t), so a pair reads one stage and DEPTH - 1 stages are in flight while
// it computes. A thread's first staged pair in its column (or one after a general-path pair) takes those twelve
// carried words from global memory.
//
// Blocks: the main columns [we, ea) of the rows [m0, m1) (split.h, staged_block_column) in tiles of 32 x TY walking a
// z-slab of level pairs, then the strip blocks (face columns) of the plain kernel. A thread whose pair is interior
// (every source fluid, both levels below the lid, not on a face) relaxes it from the stage (fast_pair_relax, the
// arithmetic of the plain paired path, so the result is bit-identical to it); otherwise each of its levels takes the
// general single-cell path from global memory.
//
// Copies: lane 0 of warp 0 arms the stage's mbarrier with the stage's byte count, then lanes 0-25 issue one box copy
// each (no multicast; this GPU's memory only). Every consumer wait is bounded by the global timer: a wait that runs
// out stops the block (its remaining cells are not stepped), thread 0 waits, bounded again, for the copies it issued,
// and the handle's error word is set, which the host turns into a lost state. A copy whose destination, barrier,
// tensor map or x coordinate is misaligned is not issued: it sets the error word instead.
#pragma once

#include "fused.cuh"
#include "tma.cuh"

namespace ahx {

// geometry of the stages of the staged paired step (32 x TY columns, 4-byte words)
template <int TY>
struct PairStage {
  static constexpr int H = 4;                 // x halo of a wide box: one 16-byte granule of words
  static constexpr int WW = 32 + 2 * H;       // wide box width (words)
  static constexpr int wide_bytes = WW * TY * 4;
  static constexpr int narrow_bytes = 32 * TY * 4;
  static constexpr int slot_cx(int slot) { return slot < 19 ? kC19[slot][0] : kC7[slot - 19][0]; }
  static constexpr int slot_cy(int slot) { return slot < 19 ? kC19[slot][1] : kC7[slot - 19][1]; }
  static constexpr int slot_cz(int slot) { return slot < 19 ? kC19[slot][2] : kC7[slot - 19][2]; }
  // byte offset of population slot s (f: q, g: 19 + q) inside a stage; each box keeps 128-byte alignment
  static constexpr int box_offset(int slot) {
    int off = 0;
    for (int s = 0; s < slot; ++s) off += slot_cx(s) != 0 ? wide_bytes : narrow_bytes;
    return off;
  }
  static constexpr int stage_bytes = box_offset(26);
  static_assert(wide_bytes % 128 == 0 && narrow_bytes % 128 == 0, "boxes keep 128-byte alignment");
};

// dynamic shared memory of the staged paired step: 128 bytes of alignment slack, DEPTH stages, a 128-byte slot for
// the DEPTH barriers, then the nz-entry float4 inflow profile
template <int TY, int DEPTH>
constexpr size_t pair_stage_smem_bytes(int nz) {
  static_assert(8 * DEPTH <= kBarSlot, "barriers fit their slot");
  return 128 + (size_t)DEPTH * PairStage<TY>::stage_bytes + kBarSlot + 16 * (size_t)nz;
}

// copy slot `lane` (0-25) of stage t into its place: the box of words the block's columns pull that population from,
// at level pair t (t + 1 for cz = -1); x0: first main column of the block, y0: its first row
template <int TY>
__device__ __forceinline__ void pair_stage_issue(const TmaMaps& M, unsigned char* stage, uint64_t* bar, int lane,
                                                 int x0, int y0, int t, int* err) {
  using G = PairStage<TY>;
  const bool isf = lane < 19;
  const int q = isf ? lane : lane - 19;
  int scx = 0, scy = 0, scz = 0, off = 0;
  // per-lane direction and box offset, from the compile-time tables
  static_for<26>([&](auto S) {
    constexpr int s = S;
    if (s == lane) {
      scx = G::slot_cx(s);
      scy = G::slot_cy(s);
      scz = G::slot_cz(s);
      off = G::box_offset(s);
    }
  });
  const int x = scx != 0 ? x0 - G::H : x0;
  if ((x & 3) != 0) {   // a box must start on a 16-byte boundary (4 words)
    atomicExch(err, 2);
    return;
  }
  const CUtensorMap* map = isf ? (scx != 0 ? &M.fw : &M.fn) : (scx != 0 ? &M.gw : &M.gn);
  tma_load_4d(stage + off, map, x, y0 - scy, scz == -1 ? t + 1 : t, q, bar, err);
}

template <class S, int TY, int DEPTH>
__device__ __forceinline__ void step_pair_tma_block(const DomainView& D, const TmaMaps& M, const StepSplit& SP,
                                                    int zslab) {
  using TF = StoreF<S>;
  using TG = StoreG<S>;
  static_assert(kLevelPairs<TF> && kLevelPairs<TG>, "the staged paired step reads level-paired 16-bit planes");
  using KF = CodecF<S>;
  using G = PairStage<TY>;
  constexpr int STAGE = G::stage_bytes;
  extern __shared__ unsigned char pst_smem_raw[];
  __shared__ ParamsHead sP;
  __shared__ int s_kmin;
  // stop flags, one per iteration parity: set before a block barrier, read after it (a flag read in iteration n is
  // written again only in iteration n + 2, after the barrier of iteration n + 1)
  __shared__ int s_abort[2];
  __shared__ uint32_t s_tkey;
  unsigned char* base =
      reinterpret_cast<unsigned char*>((reinterpret_cast<uintptr_t>(pst_smem_raw) + 127) & ~uintptr_t(127));
  uint64_t* bars = reinterpret_cast<uint64_t*>(base + (size_t)DEPTH * STAGE);
  float4* prof = reinterpret_cast<float4*>(base + (size_t)DEPTH * STAGE + kBarSlot);

  const int tx = threadIdx.x, ty = threadIdx.y;
  const int tid = ty * 32 + tx;
  const int x0 = SP.we + (int)blockIdx.x * 32, y0 = SP.m0 + (int)blockIdx.y * TY;
  const int i = x0 + tx, j = y0 + ty;
  const bool valid = i < SP.ea && j < SP.m1;
  const int k0 = (int)blockIdx.z * zslab;
  const int k1 = min(D.nz, k0 + zslab);
  if (tid < 16) reinterpret_cast<int*>(&sP)[tid] = reinterpret_cast<const int*>(D.params)[tid];
  const float4* gprof = reinterpret_cast<const float4*>(D.params + 64);
  for (int z = tid; z < D.nz; z += 32 * TY) prof[z] = gprof[z];
  if (tid == 0) {
    s_kmin = k1;
    s_abort[0] = s_abort[1] = 0;
    if constexpr (kDitherOf<S>) s_tkey = mix32(__ldcg(D.tick) * 0x9e3779b9u + 0x632be5abu);
    for (int s = 0; s < DEPTH; ++s) mbar_init(&bars[s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  const ParamsHead& P = sP;
  const RelaxConst RK = relax_const(P);
  Column<float> C;
  int kst = k1;
  if (valid) {
    load_column(D, P, i, j, C);
    kst = max(k0, C.kg);
  }
  kst = __reduce_min_sync(0xffffffffu, kst);
  if (tx == 0) atomicMin(&s_kmin, kst);
  __syncthreads();
  const int kb = s_kmin;
  if (kb >= k1) return;   // every column of the tile is solid in this slab: no copy was issued
  // pairs [pb, pe) hold the levels [kb, k1); stage s (0 .. nst - 1) is the one of pair pb + s
  const int pb = kb >> 1, pe = (k1 + 1) >> 1;
  const int nst = pe - pb;
  const int lane = tid & 31, warp = tid >> 5;
  auto issue = [&](int s) {   // warp 0: stage s into slot s % DEPTH
    unsigned char* st = base + (size_t)(s % DEPTH) * STAGE;
    uint64_t* bar = &bars[s % DEPTH];
    if (lane == 0) mbar_arm(bar, (unsigned)STAGE);
    __syncwarp();
    if (lane < 26) pair_stage_issue<TY>(M, st, bar, lane, x0, y0, pb + s, D.err);
  };
  if (warp == 0)
    for (int s = 0; s < DEPTH && s < nst; ++s) issue(s);

  const uint32_t px = (uint32_t)D.px, ps = D.ps;
  const uint32_t mc = (uint32_t)j * px + (uint32_t)i;
  uint32_t gid0 = 0, gstep = 0;
  if constexpr (kDitherOf<S>) {
    gid0 = (uint32_t)(j + D.jg0) * px + (uint32_t)i;
    gstep = (uint32_t)D.nyg * px;
  }
  auto seed = [&](int kk) -> uint32_t {
    if constexpr (kDitherOf<S>) return mix32((gid0 + (uint32_t)kk * gstep) ^ s_tkey);
    else return 0u;
  };
  // per-thread word offsets inside a box: wide boxes start H words before the block's first column
  const int owide = ty * G::WW + tx + G::H, onarrow = ty * 32 + tx;
  // the carried word of each cz != 0 population (only those entries are used): for cz = +1 word t - 1, for cz = -1
  // word t of the source column, when this thread's previous pair was staged
  uint32_t carry_f[19], carry_g[7];
  bool have_carry = false;
#pragma unroll 1
  for (int it = 0; it < nst; ++it) {
    const int t = pb + it;
    const bool ok = mbar_wait_bounded(&bars[it % DEPTH], (unsigned)((it / DEPTH) & 1), kStageWaitLimitNs);
    if (!ok) s_abort[it & 1] = 1;   // a stage that did not arrive stops the block after this pair
    const int k = 2 * t;
    const bool in2 = ok && valid && k >= C.kg && k >= k0 && !C.face && k >= C.kint && k + 1 < D.nz - 1;
    if (in2) {
      const uint32_t* s0 = reinterpret_cast<const uint32_t*>(base + (size_t)(it % DEPTH) * STAGE);
      const uint32_t nf = lvl<TF>(k, mc, ps), ng = lvl<TG>(k, mc, ps);
      if (!have_carry) {
        // first staged pair of the column here: the carried words from global memory (the pull offset of a cz = +1
        // population points at word t - 1 of its source column, of a cz = -1 population at word t)
        static_for<19>([&](auto Q) {
          constexpr int q = Q;
          if constexpr (kC19[q][2] != 0) carry_f[q] = KF::load_w(static_cast<const TF*>(D.src_f[q]) + nf);
        });
        static_for<7>([&](auto Q) {
          constexpr int q = Q;
          if constexpr (kC7[q][2] != 0) carry_g[q] = CodecG<S>::load_w(static_cast<const TG*>(D.src_g[q]) + ng);
        });
      }
      float2 f[19], g[7];
      static_for<26>([&](auto Sl) {
        constexpr int sl = Sl;
        constexpr bool isf = sl < 19;
        constexpr int q = isf ? sl : sl - 19;
        constexpr int cx = G::slot_cx(sl);
        constexpr int cz = G::slot_cz(sl);
        constexpr int wo = G::box_offset(sl) / 4 - cx;   // word offset of the box, shifted to the source column
        const uint32_t cur = s0[(cx != 0 ? owide : onarrow) + wo];
        uint32_t w = cur;
        if constexpr (cz != 0) {
          // cz = +1: (high half of word t - 1, low half of word t); cz = -1: (high of word t, low of word t + 1)
          w = __byte_perm(isf ? carry_f[q] : carry_g[q], cur, 0x5432);
          if constexpr (isf) carry_f[q] = cur;
          else carry_g[q] = cur;
        }
        if constexpr (isf) f[q] = word_dec_f<TF>(w, (float)w19(q));
        else g[q] = word_dec_g<TG>(w);
      });
      fast_pair_relax<S>(D, P, RK, prof, C, k, nf, ng, f, g, seed(k), seed(k + 1));
      have_carry = true;
    } else {
      have_carry = false;
      if (ok && valid) {
        for (int kk = max(k, max(k0, C.kg)); kk < min(k + 2, k1); ++kk) {
          const uint32_t nf = lvl<TF>(kk, mc, ps), ng = lvl<TG>(kk, mc, ps);
          Cell<float> X;
          if (!C.face && kk >= C.kint && kk < D.nz - 1) stream_interior<S>(D, prof, C, kk, mc, X);
          else stream_cell<S>(D, P, prof, C, kk, mc, X);
          Macro<float> Mm;
          fast_update<S>(D, P, RK, C, kk, nf, ng, X, Mm, seed(kk));
        }
      }
    }
    __syncthreads();   // every thread is done with stage it
    if (s_abort[it & 1]) {
      if (tid == 0) {
        atomicExch(D.err, 1);
        // wait (bounded) for the copies still in flight into this block's stages before it exits
        for (int s = it; s < min(nst, it + DEPTH); ++s)
          mbar_wait_bounded(&bars[s % DEPTH], (unsigned)((s / DEPTH) & 1), kStageWaitLimitNs);
      }
      return;
    }
    if (warp == 0 && it + DEPTH < nst) issue(it + DEPTH);
  }
}

}  // namespace ahx

// Instantiates the fused step kernels for one arithmetic variant and one population storage. step_unit.cu is compiled
// once per (variant, storage) with AHX_STEP_NS = exact (-fmad=false) or fast (-fmad=true, AHX_STEP_FAST=1) and
// AHX_STEP_PREC = the ahx_precision value of the storage, so the 14 instantiation sets compile in parallel; the
// precision switch of each variant is step_dispatch.cu.
#pragma once

#include <type_traits>

#include "fused.cuh"
#include "launch.h"
#include "tma.cuh"
#include "tma_pairs.cuh"

namespace ahx {
namespace AHX_STEP_NS {

#ifndef AHX_STEP_FAST
#define AHX_STEP_FAST 0
#endif

// MINB = 0: up to 256 threads per block, registers as the compiler likes; MINB = 4 / 5 / 6 / 8: 128-thread blocks
// with that many resident per SM (a 128 / 96 / 80 / 64 register budget), chosen by the launch-shape tuner
// Stochastic-rounding storages: a block (tile) of a step reports done; the last of the step's `blocks` to do so
// advances the step counter the next step's dithers are keyed on (every block read it before reporting).
__device__ __forceinline__ void tick_done(const DomainView& D, uint32_t blocks) {
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    if (atomicAdd(D.tick + 1, 1u) == blocks - 1) {
      atomicExch(D.tick + 1, 0u);
      atomicAdd(D.tick, 1u);
    }
  }
}

template <class S, int MODE, bool BUDGET, int MINB, bool PAIRS = false>
__global__ void __launch_bounds__(MINB ? 128 : 256, MINB ? MINB : 1) step_kernel(DomainView D, int zslab) {
  step_block<S, MODE, BUDGET, AHX_STEP_FAST != 0, PAIRS>(D, blockIdx.x, blockIdx.y, blockIdx.z, zslab);
  if constexpr (kDitherOf<S>) tick_done(D, gridDim.x * gridDim.y * gridDim.z);
}

template <class S, int TY, int DEPTH>
__global__ void __launch_bounds__(32 * TY, TY == 4 ? 4 : 2)
    step_tma_kernel(DomainView D, const __grid_constant__ TmaMaps M, int zslab) {
  step_tma_block<S, AHX_STEP_FAST != 0, TY, DEPTH>(D, M, zslab);
}

// Staged paired step of the 16-bit storages (FMA build): main blocks of 32 x TY columns read their interior pairs'
// sources from TMA-staged level-pair words (tma_pairs.cuh); the strip blocks after them run the plain paired path.
// Resident blocks per SM follow the shared memory a block takes (DEPTH stages of 14.5 KB at TY = 4, 29 KB at TY = 8)
// and set the register budget (5 / 4 / 3 blocks of 128 threads: 96 / 128 / 168 registers).
template <int TY, int DEPTH>
inline constexpr int kPairStageBlocks = TY == 8 ? 2 : (DEPTH <= 2 ? 5 : (DEPTH == 3 ? 4 : 3));
template <class S, int TY, int DEPTH>
__global__ void __launch_bounds__(32 * TY, kPairStageBlocks<TY, DEPTH>)
    step_pair_tma_kernel(DomainView D, const __grid_constant__ TmaMaps M, int zslab) {
  const StepSplit SP = step_split(D.nx, D.jlo, D.jhi, D.jbase, D.jg0, D.nyg, D.strip);
  const int mby = staged_main_blocks_y(SP, TY);
  if ((int)blockIdx.y < mby)
    step_pair_tma_block<S, TY, DEPTH>(D, M, SP, zslab);
  else
    step_block<S, 0, false, true, true>(D, blockIdx.x, (int)blockIdx.y - mby + main_blocks_y(D.jhi, D.jbase, TY),
                                        blockIdx.z, zslab);
  if constexpr (kDitherOf<S>) tick_done(D, gridDim.x * gridDim.y * gridDim.z);
}

// Batched step: one persistent launch steps every member domain of a batch. Blocks take tiles (32 x 4 columns x that
// member's z-slab) from a device counter in list order until the list is exhausted, so unequal tiles balance; a
// block fetches its next tile index while it works on the current one, and copies a member's view (and stages its
// parameters and profile) only when the tile's member differs from its previous tile's. Each tile runs the same
// step_block as a solo launch, so a member's result is bit-identical to stepping it alone. The tile count is read
// from device memory, so one captured launch serves any membership the tables describe. The last block to finish
// resets the counters for the next launch on the stream (launches on one stream do not overlap).
template <class S, int MINB, bool PAIRS>
__global__ void __launch_bounds__(128, MINB) batch_kernel(const DomainView* __restrict__ views,
                                                          const BatchTile* __restrict__ tiles,
                                                          const int* __restrict__ zslabs,
                                                          const int* __restrict__ ntiles_ptr, int* sched) {
  __shared__ DomainView sD;
  __shared__ int s_zslab, s_t, s_member;
  static_assert(sizeof(DomainView) % 4 == 0, "the view copies as 32-bit words");
  const int tid = threadIdx.y * 32 + threadIdx.x;
  const int ntiles = *ntiles_ptr;
  if (tid == 0) {
    s_member = -1;
    s_t = atomicAdd(&sched[0], 1);
  }
  __syncthreads();
  for (;;) {
    const int t = s_t;
    if (t >= ntiles) break;
    const BatchTile T = tiles[t];
    const bool fresh = (int)T.member != s_member;
    __syncthreads();   // every thread has read s_t and s_member
    if (tid == 0) s_t = atomicAdd(&sched[0], 1);   // the next tile, fetched while this one runs
    if (fresh) {
      const int* src = reinterpret_cast<const int*>(views + T.member);
      int* dst = reinterpret_cast<int*>(&sD);
      for (int w = tid; w < (int)(sizeof(DomainView) / 4); w += 128) dst[w] = src[w];
      if (tid == 0) {
        s_zslab = zslabs[T.member];
        s_member = T.member;
      }
    }
    __syncthreads();
    step_block<S, 0, false, AHX_STEP_FAST != 0, PAIRS>(sD, T.bx, T.by, T.bz, s_zslab, fresh);
    if constexpr (kDitherOf<S>) tick_done(sD, sD.tick_blocks);
    __syncthreads();   // the next tile may overwrite the view and the staged profile
  }
  if (tid == 0) {
    __threadfence();
    if (atomicAdd(&sched[1], 1) == (int)gridDim.x - 1) {
      atomicExch(&sched[0], 0);
      atomicExch(&sched[1], 0);
    }
  }
}

template <class S, int MINB, bool PAIRS>
static cudaError_t batch_t(const BatchLaunch& B, cudaStream_t s, int* occupancy) {
  const size_t smem = (size_t)B.max_nz * sizeof(float4);
  if (occupancy)
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(occupancy, batch_kernel<S, MINB, PAIRS>, 128, smem);
  batch_kernel<S, MINB, PAIRS><<<B.grid, dim3(32, 4), smem, s>>>(B.views, B.tiles, B.zslabs, B.ntiles, B.sched);
  return cudaGetLastError();
}

template <class S, bool PAIRS>
static cudaError_t batch_m(const BatchLaunch& B, cudaStream_t s, int* occupancy) {
  switch (B.minb) {
    case 5: return batch_t<S, 5, PAIRS>(B, s, occupancy);
    case 6: return batch_t<S, 6, PAIRS>(B, s, occupancy);
    default: return batch_t<S, 4, PAIRS>(B, s, occupancy);
  }
}

template <class S>
static cudaError_t batch_s(const BatchLaunch& B, cudaStream_t s, int* occupancy) {
  if constexpr (AHX_STEP_FAST != 0 && std::is_same_v<RealOf<S>, float>) {
    if (B.pairs) return batch_m<S, true>(B, s, occupancy);
  }
  return batch_m<S, false>(B, s, occupancy);
}

template <class S, int TY, int DEPTH>
static cudaError_t launch_tma_t(const DomainView& D, const StepLaunch& L, cudaStream_t s) {
  const int zs = L.zslab > 0 ? L.zslab : D.nz;
  const size_t smem = tma_smem_bytes<S, TY, DEPTH>(D.nz);
  // the dynamic shared-memory size the attribute allows, per device (an attribute is per function and device)
  static int configured[64] = {0};
  int dev = 0;
  cudaGetDevice(&dev);
  if (dev < 0 || dev >= 64 || configured[dev] < (int)smem) {
    const cudaError_t e = cudaFuncSetAttribute(step_tma_kernel<S, TY, DEPTH>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    if (dev >= 0 && dev < 64) configured[dev] = (int)smem;
  }
  dim3 block(32, TY);
  dim3 grid((D.nx + 31) / 32, (D.ny + TY - 1) / TY, (D.nz + zs - 1) / zs);
  step_tma_kernel<S, TY, DEPTH><<<grid, block, smem, s>>>(D, *L.maps, zs);
  return cudaGetLastError();
}

template <class S>
static cudaError_t launch_tma(const DomainView& D, const StepLaunch& L, cudaStream_t s) {
  const int key = L.tma_ty * 10 + L.tma_depth;
  switch (key) {
    case 42: return launch_tma_t<S, 4, 2>(D, L, s);
    case 43: return launch_tma_t<S, 4, 3>(D, L, s);
    case 44: return launch_tma_t<S, 4, 4>(D, L, s);
    case 82: return launch_tma_t<S, 8, 2>(D, L, s);
    case 83: return launch_tma_t<S, 8, 3>(D, L, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class S, int TY, int DEPTH>
static cudaError_t launch_pair_tma_t(const DomainView& D, const StepLaunch& L, cudaStream_t s) {
  if constexpr (AHX_STEP_FAST != 0) {
    int zs = L.zslab > 0 ? L.zslab : D.nz;
    zs = (zs + 1) & ~1;   // blocks start on an even level: a level pair is one word
    const size_t smem = pair_stage_smem_bytes<TY, DEPTH>(D.nz);
    static int configured[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64 || configured[dev] < (int)smem) {
      const cudaError_t e = cudaFuncSetAttribute(step_pair_tma_kernel<S, TY, DEPTH>,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      if (e != cudaSuccess) return e;
      if (dev >= 0 && dev < 64) configured[dev] = (int)smem;
    }
    if (D.strip <= 0) return cudaErrorInvalidValue;   // the staged tiles need the face columns in strip blocks
    const StepSplit SP = step_split(D.nx, D.jlo, D.jhi, D.jbase, D.jg0, D.nyg, D.strip);
    dim3 grid(SP.gx, staged_main_blocks_y(SP, TY) + strip_blocks_y(SP, TY), (D.nz + zs - 1) / zs);
    step_pair_tma_kernel<S, TY, DEPTH><<<grid, dim3(32, TY), smem, s>>>(D, *L.maps, zs);
    return cudaGetLastError();
  } else {
    return cudaErrorInvalidValue;
  }
}

template <class S>
static cudaError_t launch_pair_tma(const DomainView& D, const StepLaunch& L, cudaStream_t s) {
  switch (L.tma_ty * 10 + L.tma_depth) {
    case 42: return launch_pair_tma_t<S, 4, 2>(D, L, s);
    case 43: return launch_pair_tma_t<S, 4, 3>(D, L, s);
    case 44: return launch_pair_tma_t<S, 4, 4>(D, L, s);
    case 82: return launch_pair_tma_t<S, 8, 2>(D, L, s);
    case 83: return launch_pair_tma_t<S, 8, 3>(D, L, s);
    default: return cudaErrorInvalidValue;
  }
}

template <class S, int MODE, bool BUDGET>
static cudaError_t launch_t(const DomainView& D, const StepLaunch& L, cudaStream_t s) {
  if constexpr (MODE == 0 && !BUDGET && std::is_same_v<StoreF<S>, StoreG<S>> && !kDitherOf<S> &&
                !kLevelPairs<StoreF<S>>) {
    // the staged kernel stages f and g with one element size, one level per box: uniform round-to-nearest storages
    // of 4- and 8-byte elements only
    if (L.tma_ty > 0 && L.maps != nullptr) return launch_tma<S>(D, L, s);
  }
  if constexpr (MODE == 0 && !BUDGET && AHX_STEP_FAST != 0 && kLevelPairs<StoreF<S>> && kLevelPairs<StoreG<S>>) {
    // the staged paired step: level-paired f and g (FP16, BF16, FP16 with stochastic rounding)
    if (L.tma_ty > 0 && L.pairs && L.maps != nullptr) return launch_pair_tma<S>(D, L, s);
  }
  const int minb = (MODE == 0 && !BUDGET) ? L.minb : 0;
  const int by = minb ? 4 : (L.block_y > 0 ? L.block_y : 4);
  const int zs = L.zslab > 0 ? L.zslab : D.nz;
  dim3 block(kBlockX, by);
  // the rows [jbase, jhi) the step updates (all rows, unless a slab or a band of rows): the main blocks, then the
  // strip blocks (step_split)
  const StepSplit SP = step_split(D.nx, D.jlo, D.jhi, D.jbase, D.jg0, D.nyg, D.strip);
  dim3 grid(SP.gx, main_blocks_y(D.jhi, D.jbase, by) + strip_blocks_y(SP, by), (D.nz + zs - 1) / zs);
  const size_t smem = (size_t)D.nz * sizeof(float4);
  if constexpr (MODE == 0 && !BUDGET && AHX_STEP_FAST != 0 && std::is_same_v<RealOf<S>, float>) {
    if (L.pairs) {
      switch (minb) {
        case 4: step_kernel<S, 0, false, 4, true><<<grid, block, smem, s>>>(D, zs); return cudaGetLastError();
        case 5: step_kernel<S, 0, false, 5, true><<<grid, block, smem, s>>>(D, zs); return cudaGetLastError();
        case 6: step_kernel<S, 0, false, 6, true><<<grid, block, smem, s>>>(D, zs); return cudaGetLastError();
        case 8: step_kernel<S, 0, false, 8, true><<<grid, block, smem, s>>>(D, zs); return cudaGetLastError();
        default: step_kernel<S, 0, false, 0, true><<<grid, block, smem, s>>>(D, zs); return cudaGetLastError();
      }
    }
  }
  if constexpr (MODE == 0 && !BUDGET) {
    if (minb == 4) {
      step_kernel<S, MODE, BUDGET, 4><<<grid, block, smem, s>>>(D, zs);
      return cudaGetLastError();
    }
    if (minb == 5) {
      step_kernel<S, MODE, BUDGET, 5><<<grid, block, smem, s>>>(D, zs);
      return cudaGetLastError();
    }
    if (minb == 6) {
      step_kernel<S, MODE, BUDGET, 6><<<grid, block, smem, s>>>(D, zs);
      return cudaGetLastError();
    }
    if (minb == 8) {
      step_kernel<S, MODE, BUDGET, 8><<<grid, block, smem, s>>>(D, zs);
      return cudaGetLastError();
    }
  }
  step_kernel<S, MODE, BUDGET, 0><<<grid, block, smem, s>>>(D, zs);
  return cudaGetLastError();
}

template <class S>
static cudaError_t launch_s(const DomainView& D, const StepLaunch& L, cudaStream_t s) {
  if (L.budget) {
    switch (L.mode) {
      case 1: return launch_t<S, 1, true>(D, L, s);
      case 2: return launch_t<S, 2, true>(D, L, s);
      default: return launch_t<S, 0, true>(D, L, s);
    }
  }
  switch (L.mode) {
    case 1: return launch_t<S, 1, false>(D, L, s);
    case 2: return launch_t<S, 2, false>(D, L, s);
    default: return launch_t<S, 0, false>(D, L, s);
  }
}

// the storage type of each ahx_precision value
template <int P>
struct PrecStorage;
template <>
struct PrecStorage<0> { using T = float; };
template <>
struct PrecStorage<1> { using T = __half; };
template <>
struct PrecStorage<2> { using T = __nv_bfloat16; };
template <>
struct PrecStorage<3> { using T = double; };
template <>
struct PrecStorage<4> { using T = Mixed<__half, float>; };
template <>
struct PrecStorage<5> { using T = Mixed<__nv_bfloat16, float>; };
template <>
struct PrecStorage<6> { using T = half_sr; };

#ifdef AHX_STEP_PREC
#define AHX_PREC_CAT2(a, b) a##b
#define AHX_PREC_CAT(a, b) AHX_PREC_CAT2(a, b)
// the entry points of this translation unit's storage, called by the precision switch (step_dispatch.cu)
cudaError_t AHX_PREC_CAT(launch_step_p, AHX_STEP_PREC)(const DomainView& D, const StepLaunch& L, cudaStream_t s) {
  return launch_s<typename PrecStorage<AHX_STEP_PREC>::T>(D, L, s);
}
cudaError_t AHX_PREC_CAT(launch_batch_p, AHX_STEP_PREC)(const BatchLaunch& B, cudaStream_t s, int* occupancy) {
  return batch_s<typename PrecStorage<AHX_STEP_PREC>::T>(B, s, occupancy);
}
#endif

}  // namespace AHX_STEP_NS
}  // namespace ahx

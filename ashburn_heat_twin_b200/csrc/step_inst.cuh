// Instantiates the fused step kernels for one arithmetic variant. Included once by step_exact.cu and once by
// step_fast.cu with AHX_STEP_NS set to the variant's namespace; the two translation units are compiled with
// -fmad=false and -fmad=true respectively.
#pragma once

#include "fused.cuh"
#include "launch.h"

namespace ahx {
namespace AHX_STEP_NS {

#ifndef AHX_STEP_FAST
#define AHX_STEP_FAST 0
#endif

template <class S, int MODE, bool BUDGET>
__global__ void __launch_bounds__(256) step_kernel(DomainView D, int zslab) {
  step_block<S, MODE, BUDGET, AHX_STEP_FAST != 0>(D, blockIdx.x, blockIdx.y, blockIdx.z, zslab);
}

template <class S, int MODE, bool BUDGET>
static cudaError_t launch_t(const DomainView& D, const StepLaunch& L, cudaStream_t s) {
  const int by = L.block_y > 0 ? L.block_y : 4;
  const int zs = L.zslab > 0 ? L.zslab : D.nz;
  dim3 block(kBlockX, by);
  dim3 grid((D.nx + kBlockX - 1) / kBlockX, (D.ny + by - 1) / by, (D.nz + zs - 1) / zs);
  const size_t smem = (size_t)D.nz * sizeof(float4);
  step_kernel<S, MODE, BUDGET><<<grid, block, smem, s>>>(D, zs);
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

cudaError_t launch_step(const DomainView& D, const StepLaunch& L, cudaStream_t s) {
  switch (L.precision) {
    case 0: return launch_s<float>(D, L, s);
    case 1: return launch_s<__half>(D, L, s);
    case 2: return launch_s<__nv_bfloat16>(D, L, s);
    case 3: return launch_s<double>(D, L, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace AHX_STEP_NS
}  // namespace ahx

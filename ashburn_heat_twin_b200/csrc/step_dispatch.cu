// Precision switch of one arithmetic variant (compiled with -DAHX_STEP_NS=exact or fast): forwards to the entry
// points of the per-storage translation units (step_unit.cu compiled with AHX_STEP_PREC = 0 .. 6).
#ifndef AHX_STEP_NS
#error "step_dispatch.cu is compiled with -DAHX_STEP_NS=exact|fast"
#endif
#include "launch.h"

namespace ahx {
namespace AHX_STEP_NS {

#define AHX_STORAGE_ENTRY(p)                                                                     \
  cudaError_t launch_step_p##p(const DomainView& D, const StepLaunch& L, cudaStream_t s);       \
  cudaError_t launch_batch_p##p(const BatchLaunch& B, cudaStream_t s, int* occupancy);
AHX_STORAGE_ENTRY(0)
AHX_STORAGE_ENTRY(1)
AHX_STORAGE_ENTRY(2)
AHX_STORAGE_ENTRY(3)
AHX_STORAGE_ENTRY(4)
AHX_STORAGE_ENTRY(5)
AHX_STORAGE_ENTRY(6)
#undef AHX_STORAGE_ENTRY

cudaError_t launch_step(const DomainView& D, const StepLaunch& L, cudaStream_t s) {
  switch (L.precision) {
    case 0: return launch_step_p0(D, L, s);
    case 1: return launch_step_p1(D, L, s);
    case 2: return launch_step_p2(D, L, s);
    case 3: return launch_step_p3(D, L, s);
    case 4: return launch_step_p4(D, L, s);
    case 5: return launch_step_p5(D, L, s);
    case 6: return launch_step_p6(D, L, s);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t launch_batch(const BatchLaunch& B, cudaStream_t s, int* occupancy) {
  switch (B.precision) {
    case 0: return launch_batch_p0(B, s, occupancy);
    case 1: return launch_batch_p1(B, s, occupancy);
    case 2: return launch_batch_p2(B, s, occupancy);
    case 3: return launch_batch_p3(B, s, occupancy);
    case 4: return launch_batch_p4(B, s, occupancy);
    case 5: return launch_batch_p5(B, s, occupancy);
    case 6: return launch_batch_p6(B, s, occupancy);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace AHX_STEP_NS
}  // namespace ahx

// Fused step kernels of one arithmetic variant and one population storage. Compiled once per pair (the build passes
// AHX_STEP_NS, AHX_STEP_FAST and AHX_STEP_PREC): the exact variant with -fmad=false, so every f32 expression is
// evaluated in the reference's order with individually rounded operations; the fast variant with -fmad=true,
// approximate division and square root, and the paired relaxation of fast_update (fused.cuh).
#ifndef AHX_STEP_NS
#error "step_unit.cu is compiled with -DAHX_STEP_NS=exact|fast -DAHX_STEP_PREC=<ahx_precision>"
#endif
#include "step_inst.cuh"

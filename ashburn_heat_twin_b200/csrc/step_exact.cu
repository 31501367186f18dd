// Fused step, IEEE-exact variant: built with -fmad=false (no contraction), so every f32 expression is evaluated in the
// reference's order with individually rounded operations.
#define AHX_STEP_NS exact
#include "step_inst.cuh"

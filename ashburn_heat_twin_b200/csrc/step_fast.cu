// Fused step, contracted variant: built with -fmad=true and approximate division / square root
// (-prec-div=false -prec-sqrt=false), and the paired collision of fast_update (fused.cuh).
#define AHX_STEP_NS fast
#define AHX_STEP_FAST 1
#include "step_inst.cuh"

// Fused step, contracted variant: built with -fmad=true (multiply-adds fused into FMA).
#define AHX_STEP_NS fast
#include "step_inst.cuh"

// FP64 engine instantiation (compiled with --fmad=false: every operation
// individually rounded, as in the CPU restatement).
#include "engine.cuh"

XFB_INSTANTIATE_ENGINE(double)

// FP32 engine instantiation (compiled with FMA contraction).
#include "engine.cuh"

XFB_INSTANTIATE_ENGINE(float)

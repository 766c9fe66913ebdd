// Kernel set for f32 transforms of length 32.
#include "kernel_set.cuh"
AZB_INSTANTIATE(float, f32, 32)

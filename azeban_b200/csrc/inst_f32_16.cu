// Kernel set for f32 transforms of length 16.
#include "kernel_set.cuh"
AZB_INSTANTIATE(float, f32, 16)

// Kernel set for f32 transforms of length 6.
#include "kernel_set.cuh"
AZB_INSTANTIATE(float, f32, 6)

// Kernel set for f32 transforms of length 192.
#include "kernel_set.cuh"
AZB_INSTANTIATE(float, f32, 192)

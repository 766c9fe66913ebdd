// Kernel set for f32 transforms of length 1024.
#include "kernel_set.cuh"
AZB_INSTANTIATE(float, f32, 1024)

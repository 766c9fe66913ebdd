// Kernel set for f64 transforms of length 128.
#include "kernel_set.cuh"
AZB_INSTANTIATE(double, f64, 128)

// Kernel set for f64 transforms of length 24.
#include "kernel_set.cuh"
AZB_INSTANTIATE(double, f64, 24)

// Kernel set for f64 transforms of length 256.
#include "kernel_set.cuh"
AZB_INSTANTIATE(double, f64, 256)

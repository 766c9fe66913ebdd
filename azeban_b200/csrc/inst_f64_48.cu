// Kernel set for f64 transforms of length 48.
#include "kernel_set.cuh"
AZB_INSTANTIATE(double, f64, 48)

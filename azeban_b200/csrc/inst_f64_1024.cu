// Kernel set for f64 transforms of length 1024.
#include "kernel_set.cuh"
AZB_INSTANTIATE(double, f64, 1024)

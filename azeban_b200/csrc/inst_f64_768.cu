// Kernel set for f64 transforms of length 768.
#include "kernel_set.cuh"
AZB_INSTANTIATE(double, f64, 768)

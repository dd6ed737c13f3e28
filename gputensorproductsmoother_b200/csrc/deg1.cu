// Kernels and launch table of polynomial degree 1.
#define TPS_DEGREE 1
#include "kernels_impl.cuh"

// Kernels and launch table of polynomial degree 2.
#define TPS_DEGREE 2
#include "kernels_impl.cuh"

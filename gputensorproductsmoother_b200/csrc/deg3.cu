// Kernels and launch table of polynomial degree 3.
#define TPS_DEGREE 3
#include "kernels_impl.cuh"

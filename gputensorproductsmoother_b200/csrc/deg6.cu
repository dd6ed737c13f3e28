// Kernels and launch table of polynomial degree 6.
#define TPS_DEGREE 6
#include "kernels_impl.cuh"

// Kernels and launch table of polynomial degree 4.
#define TPS_DEGREE 4
#include "kernels_impl.cuh"

// Kernels and launch table of polynomial degree 5.
#define TPS_DEGREE 5
#include "kernels_impl.cuh"

// Kernels and launch table of polynomial degree 7.
#define TPS_DEGREE 7
#include "kernels_impl.cuh"

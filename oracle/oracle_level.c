/*
 * TEST INFRASTRUCTURE ONLY -- instantiates the oracle's level operations in
 * FP64 (_d) and FP32 (_f).  Parity status: UNPINNED (see oracle.h).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "oracle.h"

#define CAT_(a, b) a##b
#define CAT(a, b) CAT_(a, b)

#define REAL double
#define SUF _d
#include "oracle_level.inc"
#undef REAL
#undef SUF

#define REAL float
#define SUF _f
#include "oracle_level.inc"
#undef REAL
#undef SUF

// Fused iteration kernels for the f16 state with the exact arithmetic: every
// compiled tile shape of K = 2 .. 6 (a translation unit of its own so that the
// build compiles the kernel variants in parallel).
#include "fused_launch.cuh"

POTTS_FUSED_INSTANCES(2, __half, false);
POTTS_FUSED_INSTANCES(3, __half, false);
POTTS_FUSED_INSTANCES(4, __half, false);
POTTS_FUSED_INSTANCES(5, __half, false);
POTTS_FUSED_INSTANCES(6, __half, false);

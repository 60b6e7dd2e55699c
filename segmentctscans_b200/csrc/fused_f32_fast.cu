// Fused iteration kernels for the f32 state with the fast arithmetic: every
// compiled tile shape of K = 2 .. 6 (a translation unit of its own so that the
// build compiles the kernel variants in parallel).
#include "fused_launch.cuh"

POTTS_FUSED_INSTANCES(2, float, true);
POTTS_FUSED_INSTANCES(3, float, true);
POTTS_FUSED_INSTANCES(4, float, true);
POTTS_FUSED_INSTANCES(5, float, true);
POTTS_FUSED_INSTANCES(6, float, true);

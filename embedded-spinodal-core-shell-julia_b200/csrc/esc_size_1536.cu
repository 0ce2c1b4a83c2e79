// Kernel sets for the 1536 x 1536 grid (FP64 drop-in and mixed precision).
#include "esc_dispatch.cuh"

ESC_DEFINE_SIZE(1536)

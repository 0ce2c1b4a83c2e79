// Kernel sets for the 384 x 384 grid (FP64 drop-in and mixed precision).
#include "esc_dispatch.cuh"

ESC_DEFINE_SIZE(384)

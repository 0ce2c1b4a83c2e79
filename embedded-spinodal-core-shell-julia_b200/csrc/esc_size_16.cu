// Kernel sets for the 16 x 16 grid (FP64 drop-in and mixed precision).
#include "esc_dispatch.cuh"

ESC_DEFINE_SIZE(16)

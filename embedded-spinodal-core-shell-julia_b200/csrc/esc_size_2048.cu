// Kernel sets for the 2048 x 2048 grid (FP64 drop-in and mixed precision).
#include "esc_dispatch.cuh"

ESC_DEFINE_SIZE(2048)

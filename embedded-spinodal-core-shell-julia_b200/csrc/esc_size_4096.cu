// Kernel sets for the 4096 x 4096 grid (FP64 drop-in and mixed precision).
#include "esc_dispatch.cuh"

ESC_DEFINE_SIZE(4096)

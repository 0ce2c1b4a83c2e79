// Kernel sets for the 128 x 128 grid (FP64 drop-in and mixed precision).
#include "esc_dispatch.cuh"

ESC_DEFINE_SIZE(128)

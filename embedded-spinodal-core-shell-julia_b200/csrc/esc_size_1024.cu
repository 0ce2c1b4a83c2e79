// Kernel sets for the 1024 x 1024 grid (FP64 drop-in and mixed precision).
#include "esc_dispatch.cuh"

ESC_DEFINE_SIZE(1024)

// Kernel sets for the 3072 x 3072 grid (FP64 drop-in and mixed precision).
#include "esc_dispatch.cuh"

ESC_DEFINE_SIZE(3072)

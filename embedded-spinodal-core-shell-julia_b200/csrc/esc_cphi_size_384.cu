// Coupled c-phi kernel set for axis length 384 (FP64).
#include "esc_cphi.cuh"

ESC_CPHI_DEFINE_SIZE(384)

// Fused x pass launchers, FP32 transforms.
#include "xpass.cuh"

H3D_XPASS_INSTANTIATE(float)

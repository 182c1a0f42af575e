// Fused x pass launchers, FP64 transforms.
#include "xpass.cuh"

H3D_XPASS_INSTANTIATE(double)

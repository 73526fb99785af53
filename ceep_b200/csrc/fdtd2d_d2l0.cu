// Fused 2D step kernels with two Debye poles (ND = 2, NL = 0).
#include "fdtd2d_kernels.cuh"

CEEP_FDTD2D_INSTANTIATE(2, 0)

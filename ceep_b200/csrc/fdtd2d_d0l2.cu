// Fused 2D step kernels with two Lorentz poles (ND = 0, NL = 2).
#include "fdtd2d_kernels.cuh"

CEEP_FDTD2D_INSTANTIATE(0, 2)

// Fused 2D step kernels with one Lorentz pole (ND = 0, NL = 1).
#include "fdtd2d_kernels.cuh"

CEEP_FDTD2D_INSTANTIATE(0, 1)

// Fused 2D step kernels with one Debye and one Lorentz pole (ND = 1, NL = 1).
#include "fdtd2d_kernels.cuh"

CEEP_FDTD2D_INSTANTIATE(1, 1)

// Fused 2D step kernels with one Debye pole (ND = 1, NL = 0).
#include "fdtd2d_kernels.cuh"

CEEP_FDTD2D_INSTANTIATE(1, 0)

// Fused 2D step kernels without dispersion (ND = 0, NL = 0).
#include "fdtd2d_kernels.cuh"

CEEP_FDTD2D_INSTANTIATE(0, 0)

// Parameters of the batched 3D adjoint (transposed) step kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fdtd3d.cuh"

namespace ceep {

struct Adjoint3dParams {
  Fdtd3dParams f;     // geometry, coefficients, sources, probes of the forward plan
  int zsegs_h, zsegs_e;
  long long cs;       // float4 stride between the three components of mu / nu / a saved slot
  long long icells;   // interior E cells (the gradient plane)
  int ks;             // gradient slots per cell: ca, cb, then k2 of each Debye pole
  // adjoint state, updated in place, each (3, G, nz, ny, nx, L) float4
  float4* mu;         // adjoint of E^{n+1} plus sum_q (k2_q/dt) * adjoint of J_q^{n+1}
  float4* nu;         // adjoint of H^{n+1/2} before the da factor of the next H update
  float4* lj;         // adjoint Debye currents, the forward J layout (G, poles, 3, nz, ny, nx, L)
  double* g;          // (G, ks, nzi, nyi, nxi) per-cell gradients summed over steps and TX
  const float* probe_grad;  // (ntx, nprobe, nsteps) dLoss/dprobe
};

// One adjoint step for forward step `step`.  e_n / e_np1 are the forward E
// components before and after the step as the forward's save pass wrote them
// ((3, G, nz, ny, nx, L) each): e_np1 holds the E update before the source
// was added, and so does e_n unless `e_n_post` (a copy of the state itself,
// source included: the first slot of a segment).
cudaError_t adjoint3d_launch_step(const Adjoint3dParams& a, int step, const float4* e_n, const float4* e_np1,
                                  bool e_n_post, cudaStream_t s);

}  // namespace ceep

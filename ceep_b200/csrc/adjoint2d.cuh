// Parameters of the fused 2D adjoint (transposed) step kernel.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fdtd2d.cuh"

namespace ceep {

struct Adjoint2dParams {
  Fdtd2dParams f;       // geometry, coefficients, CPML profile, sources, probes of the forward plan
  int rows;             // rows of the column segment one block walks
  int frame[4];         // frame tile columns left/right and rows top/bottom (launch order: frame tiles first)
  int smem;             // dynamic shared memory per block
  // adjoint state, every array ping-pong (read [p], write [p ^ 1]) with the
  // layouts of the forward state
  float4* ez[2];
  float4* hx[2];
  float4* hy[2];
  float4* psi_hx[2];    // y strips
  float4* psi_hy[2];    // x strips
  float4* psi_ezx[2];
  float4* psi_ezy[2];
  float4* j[2];         // (G, poles, ny, nx, L), Debye poles first, then Lorentz
  float4* jp[2];        // (G, n_lorentz, ny, nx, L): adjoint of the Lorentz J_prev
  // per-cell parameter gradients of each TX group, summed over steps:
  // (G, ny, nx, KP) with KP = 2 + 3*poles rounded up to even; per cell ca, cb,
  // then per Debye pole k1, k2, gamma and per Lorentz pole k1, k2, k3 (only
  // k2 is formed for Lorentz poles), and a zero pad
  double* g;
  const float* probe_grad;  // (ntx, nprobe, nsteps) dLoss/dprobe
  int grad_tau;             // also d/dk1 and d/dgamma (reads the forward J^n); else those slots stay 0
};

__host__ __device__ constexpr int adjoint2d_grad_width(int poles) { return (2 + 3 * poles + 1) & ~1; }

// Kernel attributes and rows per block (when a.rows == 0).
cudaError_t adjoint2d_configure(Adjoint2dParams& a);
// One adjoint step for forward step `step`: reads the adjoint of the state
// after the step from buffer `par`, writes the adjoint of the state before it
// into buffer `par ^ 1`.  ez_n / ez_np1 / j_n are the forward Ez before and
// after the step and J before it (layout of the forward fields).
cudaError_t adjoint2d_launch_step(const Adjoint2dParams& a, int step, int par, const float4* ez_n,
                                  const float4* ez_np1, const float4* j_n, cudaStream_t s);

}  // namespace ceep

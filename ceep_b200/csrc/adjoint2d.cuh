// Parameters of the 2D adjoint (transposed) step kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include "fdtd2d.cuh"

namespace ceep {

struct Adjoint2dParams {
  Fdtd2dParams f;       // geometry, coefficients, CPML profile, sources, probes of the forward plan
  // adjoint state (same layouts as the forward state)
  float4* ez;           // in place
  float4* hx[2];        // ping-pong
  float4* hy[2];
  float4* psi_hx[2];    // ping-pong (y strips)
  float4* psi_hy[2];    // ping-pong (x strips)
  float4* psi_ezx;      // in place
  float4* psi_ezy;      // in place
  float4* j;            // in place, (G, poles, ny, nx, L)
  // scratch written by the E-phase kernel and read by the H-phase kernel
  float4* cy;           // adjoint of curl_y = Hy(x) - Hy(x-1)
  float4* cx;           // adjoint of curl_x = Hx(y) - Hx(y-1)
  float4* elin;         // pointwise part of the E adjoint
  // per-cell parameter gradients, summed over transmit events and steps
  double* g;            // (2 + 3*poles, ny, nx): ca, cb, then per pole k1, k2, gamma
  const float* probe_grad;  // (ntx, nprobe, nsteps) dLoss/dprobe
};

// One adjoint step for forward step `step`: reads the adjoint of the state
// after the step, writes the adjoint of the state before it.  ez_n / ez_np1 /
// j_n are the forward Ez before and after the step and J before it (layout of
// the forward fields).  `par` is the adjoint H ping-pong buffer to read.
cudaError_t adjoint2d_launch_step(const Adjoint2dParams& a, int step, int par, const float4* ez_n,
                                  const float4* ez_np1, const float4* j_n, cudaStream_t s);

}  // namespace ceep

// Parameters of the fused 2D step kernel (device pointers, float4 = 4 TX).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ceep {

constexpr int kThreads2d = 128;

struct Fdtd2dParams {
  int nx, ny, n;
  int ntx;              // real transmit events
  int lanes;            // float4 per cell (ntx_pad / 4)
  int lanes_per_group;  // float4 per cell handled by one block (grid.z = lanes / this)
  int nprobe, nsteps;
  int n_debye, n_lorentz;
  int rows;             // rows of the column segment walked by one thread
  float db, db_dx, inv_dx, dt;
  float4* ez[2];
  float4* hx[2];
  float4* hy[2];
  float4* psi_hy[2];
  float4* psi_hx[2];
  float4* psi_ezx;
  float4* psi_ezy;
  float4* j;
  float4* j_prev;
  const float* coef;
  const float* dteps;
  const float* ade_coef;
  const float* cpml_b;
  const float* cpml_c;
  const int32_t* src_xy;
  const int32_t* prb_xy;
  const uint8_t* row_flags;
  const float* waveform;
  float* probes;
};

// Launch one step reading buffer `par` and writing buffer `par ^ 1`.
cudaError_t fdtd2d_launch_step(const Fdtd2dParams& p, int step, int par, cudaStream_t s);

}  // namespace ceep

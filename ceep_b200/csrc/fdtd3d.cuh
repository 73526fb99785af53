// Parameters of the batched 3D kernels (device pointers, float4 = 4 TX).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ceep {

struct Fdtd3dParams {
  int nx, ny, nz, n;
  int ntx, L, groups;
  int nprobe, nsteps;
  int n_debye, n_lorentz;
  int zrows, zsegs, zsegs_e;   // z segment length; segments for the H and E grids
  int zrows_shell;              // z walk length of the H shell launch
  float inv_dx, dt, inv_dt;
  long long gs_field, gs_px, gs_py, gs_pz, gs_j, gs_jp;  // per-group strides (float4)
  float4 *ex, *ey, *ez, *hx, *hy, *hz;
  float4 *psi_hxy, *psi_hzy;   // x faces (G, nz, ny, 2n, L)
  float4 *psi_hyx, *psi_hzx;   // y faces (G, nz, 2n, nx, L)
  float4 *psi_hxz, *psi_hyz;   // z faces (G, 2n, ny, nx, L)
  float4 *j, *j_prev;
  const float* coef;           // (nz, ny, nx) float4: da, db, ca, cb
  const float* ade_coef;       // (poles, nz, ny, nx) float4
  const float* cpml_b;
  const float* cpml_c;
  const int32_t* src_xyz;
  const int32_t* prb_xyz;
  const float* waveform;
  float* probes;
  // optional: the E half-step also stores each updated component (before the
  // source) of step s into slot s + 1 - save_base of save_e, a
  // (slots, 3, G, nzi, nyi, nxi, L) array over the interior E box
  // [n+1, N-n)^3 (the only cells it updates); save_cs = G * interior cells * L
  float4* save_e;
  long long save_cs;
  int save_base;
  // nonzero: the H half-step skips every cell outside [n, N-n)^3 (the CPML
  // shell and its psi), which no interior E or probe value depends on
  int interior_only;
};

// A second stream for the shell of the H half-step, with the events that
// fork it from and join it back to the step's stream.
struct Fdtd3dSide {
  cudaStream_t stream;
  cudaEvent_t fork, join;
};

// One step on stream s; with `side`, the H shell runs on side->stream beside
// the H box (both only read E and write disjoint H cells and psi).
cudaError_t fdtd3d_launch_step(const Fdtd3dParams& p, int step, cudaStream_t s, const Fdtd3dSide* side = nullptr);

}  // namespace ceep

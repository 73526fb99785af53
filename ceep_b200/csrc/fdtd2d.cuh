// Parameters of the fused 2D step kernel (device pointers, float4 = 4 TX).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace ceep {

// Consumer threads of a 2D step block (one float4 lane each); one producer
// warp more makes the block.
constexpr int kConsumers = 128;

struct Fdtd2dParams {
  int nx, ny, n;
  int ntx;              // real transmit events
  int L;                // float4 per cell inside one TX group (1, 2, 4, 8)
  int groups;           // TX groups (grid.z); all per-TX arrays are (group, ...)
  int nprobe, nsteps;
  int n_debye, n_lorentz;
  int rows;             // rows of the column segment one block walks
  int smem;             // dynamic shared memory per block
  int rows2, smem2;     // the same for the two-step kernel
  int frame1[4];        // frame tile columns left/right and rows top/bottom, one-step geometry
  int frame2[4];        // the same for the two-step geometry (launch order: frame tiles first)
  int rows_fixed;       // tile height the caller asked for (0 = chosen per kernel)
  int ntiles2;          // tiles of the two-step geometry per TX group
  int nframe2;          // its frame tiles (the first nframe2 of the frame-first order)
  int fpieces2;         // blocks (row pieces) per frame tile of the two-step kernel
  int smem2i;           // dynamic shared memory of the interior-tile two-step kernel
  int split2;           // run the two-step frame and interior tiles as two kernels (given a side stream; off by default)
  float db, db_dx, inv_dx, dt, inv_dt;
  // per-group strides in float4
  long long gs_field, gs_psi_x, gs_psi_y, gs_j, gs_jp;
  float4* ez[2];
  float4* hx[2];
  float4* hy[2];
  float4* psi_hy[2];
  float4* psi_hx[2];
  float4* psi_ezx[2];
  float4* psi_ezy[2];
  float4* j[2];
  float4* j_prev[2];
  const float* coef;      // (ny, nx) float4: ca, cb, dt/(eps_r eps0), 0
  const float* ade_coef;  // (poles, ny, nx) float4
  const float* cpml_b;
  const float* cpml_c;
  const int32_t* src_xy;
  const int32_t* prb_xy;
  const uint8_t* row_flags;
  const float* waveform;
  float* probes;
  int* status;
  // optional per-step save of Ez^{n+1} and J^{n+1} for the adjoint: slot
  // (step + 1 - save_base) of arrays shaped like (slots, whole Ez) / (slots, whole J)
  float4* save_ez;
  float4* save_j;
  int save_base;
  // Failure injection for tests of the bounded waits: the producer of every
  // block issues no copies (and no arrival) for this row, so the waits on it
  // expire.  -1 = none (the default).
  int fault_row;
  // Bound of every mbarrier wait, in ns of the global timer (0 = 1 s).
  unsigned long long wait_ns;
};

// Record an error code in the plan's status word; the first error wins.
__device__ __forceinline__ void record_status(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

// The second stream of a split two-step launch (fdtd2d_launch_step2) and
// the events that fork it from and join it back to the launching stream.
struct Fdtd2dSide {
  cudaStream_t stream;
  cudaEvent_t fork, join;
};

// Scan Ez (nf4 float4) and probes[tx][q][steps s0..s1) for NaN/Inf; on a hit
// record CEEP_ERR_NONFINITE in *status (first error wins).
cudaError_t finite_check_launch(const float4* ez, long long nf4, const float* probes, int ntx, int nprobe,
                                int nsteps, int s0, int s1, int* status, cudaStream_t s);

// One tile of a packed multi-phantom launch.
struct PackTile {
  int phantom;  // index into the parameter array
  int x0, y0;   // first cell column and row of the tile
  int g;        // TX group
  int rows;     // rows of the tile (two-step tables: a frame tile's row piece)
};

// Launch one step (two steps when `two`: tiles of the two-step geometry,
// x0 = the first thread column) of the tiles tiles_a[0, na) followed by
// tiles_b[0, nb) (all of one lane width L and one ADE shape: the running
// phantoms' frame tiles, then their interior tiles), each block reading its
// phantom's parameters from `params`; `par` is the read half of every
// ping-pong array.
cudaError_t fdtd2d_launch_packed(int L, int n_debye, int n_lorentz, const PackTile* tiles_a, int na,
                                 const PackTile* tiles_b, int nb, const Fdtd2dParams* params, int step, int par,
                                 bool two, cudaStream_t s);
int fdtd2d_cells_per_block(int L);
// Rows per block for a column-strip x row-segment grid of `slots` resident blocks.
int choose_rows(int nx, int ny, int groups, int cells_per_block, long slots, int max_rows);

// Set the kernel attributes and (if rows == 0) choose rows per block.
cudaError_t fdtd2d_configure(Fdtd2dParams& p);
// Launch one step reading buffer `par` and writing buffer `par ^ 1`.
cudaError_t fdtd2d_launch_step(const Fdtd2dParams& p, int step, int par, cudaStream_t s);
// Launch steps `step` and `step + 1` as one temporal block of two, reading
// buffer `par` and writing buffer `par ^ 1` (and the adjoint's saved Ez/J of
// both steps when the save pointers are set).  With `side` and p.split2 the
// frame tiles run as one kernel on side->stream beside the interior tiles'
// kernel on s (joined back to s before the call returns); otherwise one kernel.
cudaError_t fdtd2d_launch_step2(const Fdtd2dParams& p, int step, int par, cudaStream_t s,
                                const Fdtd2dSide* side = nullptr);

}  // namespace ceep

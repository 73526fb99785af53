// Fused 2D TMz batched FDTD step for sm_100a, TMA-pipelined.
//
// One launch advances every transmit event by one full time step:
//   H phase   interior Hx/Hy + graded-CPML psi recurrences on the four strips
//   E phase   interior Ez (+ Debye/Lorentz ADE currents) + E-CPML strip terms
//   epilogue  edge zeroing, soft source, probe record
// with exactly the per-cell region semantics of the reference's
// BatchedFDTD2D.run() (src/ceep/solvers/fdtd_2d_batched.py:454-526):
//   Hx: interior on x in [n, nx-n), y in [n, ny-1); y strips (y < n, and
//       ny-n <= y < ny-1) then apply  Hx -= db*psi  on top (double update on
//       the far strip); everything else is never updated.
//   Hy: interior on x in [n, nx-1), y in [n, ny-n); x strips x < n and
//       nx-n <= x < nx-1 apply  Hy += db*psi.
//   Ez: interior (ca, cb) on x in [n+1, nx-n), y in [n+1, ny-n); columns
//       1..n and nx-n..nx-1 (rows >= 1) get  +dt/(eps_r eps0)*psi_x, rows
//       1..n and ny-n..ny-1 (columns >= 1) get  -dt/(eps_r eps0)*psi_y, with no
//       ca factor; then the four edges are zeroed, the source added, probes read.
//
// Layout: every per-TX array is (group, y, x, L float4) with tx innermost, so
// one float4 holds four transmit events of one cell; a group is <= 32 TX.
// Per-cell coefficients (ca, cb, dt/eps; ADE k's) are one float4 per cell and
// serve every transmit event of that cell.
//
// Schedule: a block owns a column strip of CX cells and a segment of rows.
// One producer thread streams each row's slices -- Ez with a one-cell halo on
// both sides, Hx, Hy with the left halo, coefficients, ADE currents, and the
// CPML psi slices where the block touches a strip -- from HBM into a
// kStages-deep shared-memory ring with 1D bulk copies (cp.async.bulk,
// completion counted on an mbarrier).  128 consumer threads walk the rows
// upward, one float4 each, carrying Hx(x, y-1) in registers; every operand
// they read comes from shared memory, every result goes straight to HBM with
// coalesced 16-byte stores.  Hy(x-1, y) is recomputed from the staged Ez halo
// instead of being exchanged.  Every state array (fields, psi, ADE currents)
// is ping-pong buffered (read [p], write [p^1]), so a block may read any
// neighbour's old values while the neighbour writes its new ones.
//
// Every mbarrier wait is bounded in time; on expiry the block records
// CEEP_ERR_TIMEOUT in the status word, lets its copies in flight land, and
// returns.
//
// The kernels themselves are in fdtd2d_kernels.cuh, compiled once per ADE
// shape (fdtd2d_d<ND>l<NL>.cu); this file holds the run-time dispatch over
// the shapes, the rows-per-block choice and the NaN/Inf sentinel.
#include "../../include/ceep_b200.h"
#include "common.cuh"
#include "fdtd2d.cuh"

namespace ceep {

// Configure (what = 0), one step (1) or two steps (2) of one ADE shape, and
// the packed launch of one ADE shape; instantiated in fdtd2d_d<ND>l<NL>.cu.
template <int ND, int NL>
cudaError_t fdtd2d_dispatch_poles(Fdtd2dParams& p, int step, int par, cudaStream_t s, int what,
                                  const Fdtd2dSide* side);
template <int ND, int NL>
cudaError_t fdtd2d_packed_poles(int L, const PackTile* ta, int na, const PackTile* tb, int nb,
                                const Fdtd2dParams* params, int step, int par, bool two, cudaStream_t s);

// The segment length: the largest with about three waves of blocks (the
// consumers are latency-bound, so the block scheduler overlapping and
// balancing many short segments beats one wave of long ones: 600x600x16 with
// one step per launch 27 rows (one wave) 46.5 us, 10 rows 41.9 us; two steps
// per launch 27 rows 38.4 us, 8 rows 33.3 us), and at least 8 rows so the
// neighbour rows every segment loads stay a small overhead.
int choose_rows(int nx, int ny, int groups, int cells_per_block, long slots, int max_rows) {
  const long xb = (nx + cells_per_block - 1) / cells_per_block;
  const long want = 3 * slots;
  for (int rows = max_rows; rows > 8; --rows)
    if (xb * ((ny + rows - 1) / rows) * groups >= want) return rows;
  return max_rows < 8 ? max_rows : 8;
}

cudaError_t fdtd2d_launch_packed(int L, int n_debye, int n_lorentz, const PackTile* tiles_a, int na,
                                 const PackTile* tiles_b, int nb, const Fdtd2dParams* params, int step, int par,
                                 bool two, cudaStream_t s) {
  if (na + nb <= 0) return cudaSuccess;
  switch (n_debye * 3 + n_lorentz) {
    case 0: return fdtd2d_packed_poles<0, 0>(L, tiles_a, na, tiles_b, nb, params, step, par, two, s);
    case 1: return fdtd2d_packed_poles<0, 1>(L, tiles_a, na, tiles_b, nb, params, step, par, two, s);
    case 2: return fdtd2d_packed_poles<0, 2>(L, tiles_a, na, tiles_b, nb, params, step, par, two, s);
    case 3: return fdtd2d_packed_poles<1, 0>(L, tiles_a, na, tiles_b, nb, params, step, par, two, s);
    case 4: return fdtd2d_packed_poles<1, 1>(L, tiles_a, na, tiles_b, nb, params, step, par, two, s);
    case 6: return fdtd2d_packed_poles<2, 0>(L, tiles_a, na, tiles_b, nb, params, step, par, two, s);
    default: return cudaErrorInvalidValue;
  }
}

int fdtd2d_cells_per_block(int L) { return kConsumers / L; }

// NaN/Inf sentinel: grid-stride scans of Ez and of the probe samples of steps
// [s0, s1); x != x is true only for NaN, and |x| > FLT_MAX only for Inf.
__global__ void __launch_bounds__(256) finite_check_kernel(const float4* __restrict__ ez, long long nf4,
                                                           const float* __restrict__ probes, int ntx, int nprobe,
                                                           int nsteps, int s0, int s1, int* status) {
  const long long stride = (long long)gridDim.x * blockDim.x;
  const long long t0 = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  bool bad = false;
  for (long long i = t0; i < nf4; i += stride) {
    const float4 v = ez[i];
    const float m = fmaxf(fmaxf(fabsf(v.x), fabsf(v.y)), fmaxf(fabsf(v.z), fabsf(v.w)));
    bad |= !(m <= 3.4028235e38f);  // false for NaN and Inf
  }
  const int w = s1 - s0;
  const long long np = (long long)ntx * nprobe * (w > 0 ? w : 0);
  for (long long i = t0; i < np; i += stride) {
    const long long row = i / w;
    const float v = probes[row * nsteps + s0 + i % w];
    bad |= !(fabsf(v) <= 3.4028235e38f);
  }
  if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) record_status(status, CEEP_ERR_NONFINITE);
}

cudaError_t finite_check_launch(const float4* ez, long long nf4, const float* probes, int ntx, int nprobe,
                                int nsteps, int s0, int s1, int* status, cudaStream_t s) {
  if (!status) return cudaSuccess;
  finite_check_kernel<<<2 * 148, 256, 0, s>>>(ez, nf4, probes, ntx, nprobe, nsteps, s0, s1, status);
  return cudaGetLastError();
}

static cudaError_t dispatch(Fdtd2dParams& p, int step, int par, cudaStream_t s, int what,
                            const Fdtd2dSide* side = nullptr) {
  switch (p.n_debye * 3 + p.n_lorentz) {
    case 0: return fdtd2d_dispatch_poles<0, 0>(p, step, par, s, what, side);
    case 1: return fdtd2d_dispatch_poles<0, 1>(p, step, par, s, what, side);
    case 2: return fdtd2d_dispatch_poles<0, 2>(p, step, par, s, what, side);
    case 3: return fdtd2d_dispatch_poles<1, 0>(p, step, par, s, what, side);
    case 4: return fdtd2d_dispatch_poles<1, 1>(p, step, par, s, what, side);
    case 6: return fdtd2d_dispatch_poles<2, 0>(p, step, par, s, what, side);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t fdtd2d_configure(Fdtd2dParams& p) { return dispatch(p, 0, 0, nullptr, 0); }

cudaError_t fdtd2d_launch_step(const Fdtd2dParams& p, int step, int par, cudaStream_t s) {
  Fdtd2dParams q = p;
  return dispatch(q, step, par, s, 1);
}

cudaError_t fdtd2d_launch_step2(const Fdtd2dParams& p, int step, int par, cudaStream_t s, const Fdtd2dSide* side) {
  Fdtd2dParams q = p;
  return dispatch(q, step, par, s, 2, side);
}

}  // namespace ceep


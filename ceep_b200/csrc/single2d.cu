// Non-batched 2D FDTD (TMz / TEz) with CFS-CPML, PEC and Mur boundaries, for
// sm_100a: the reference's FDTD2D.step() (src/ceep/solvers/fdtd_base.py:158-190,
// src/ceep/solvers/fdtd_2d.py:111-260, src/ceep/boundaries/absorbing.py).
//
// One step is
//   step kernel  two launches, the interior blocks (no CPML code) and the
//                frame of blocks around them; warps walk 31-column strips
//                row by row: the H update of
//                every cell with its CPML H corrections (absorbing.py:332-451;
//                they read only E), then the E update of the cell from H in
//                registers (neighbours by shuffle), the soft sources of E
//                components at the cell (list order) and the boundary
//                operations in list order: CPML E corrections
//                (absorbing.py:453-561) and PEC zeroing (absorbing.py:58-72).
//                Fields and the H psi are ping-pong buffered (read [cur],
//                write [cur ^ 1]); the E psi is updated in place.
//   Hz-source  one thread adds TEz Hz sources in list order (Hz is read by
//              the neighbours' E updates, so it cannot be added inside the
//              E kernel)
//   Mur        one block: the first-order Mur update of the four edges of Ez
//              (TMz) or Hz (TEz) in the reference's order, x faces then y
//              faces (absorbing.py:126-166); last boundary operation only
//   record     probe / monitor cells into (nrec, nsteps), and a copy of the
//              snapshot field every snap_interval steps
// Fields are (nx, ny) FP32 with y fastest, the reference's layout; a step
// reads and writes each field and reads each coefficient pair once.  A run
// of steps asked for a second time is captured into a CUDA graph and replayed.
#include <map>
#include <set>
#include <tuple>

#include "../../include/ceep_b200.h"
#include "capi_internal.h"
#include "common.cuh"

namespace ceep {

struct Single2dParams {
  int nx, ny, mode, nsteps;
  float inv_dx, inv_dy, dt_mu0, dt_eps0, mur_kx, mur_ky;
  float* f[3][2];     // ping-pong fields: read [cur], write [cur ^ 1]
  const float2* ce;   // ca, cb
  const float2* ch;   // da, db
  int n_ops, ops[4];
  int t;
  const float* cpml;  // be_x, ce_x, bh_x, ch_x, be_y, ce_y, bh_y, ch_y: t each
  float* psi_e;       // x-lo, x-hi (t, ny) each, then y-lo, y-hi (nx, t) each; updated in place
  float* psi_h[2];    // same layout, ping-pong (neighbour tiles recompute from the read half)
  float* mur_prev;    // two sets of (ny, ny, nx, nx)
  int nsrc;
  const int* src;      // (nsrc, 3) x, y, field, sorted by x (stable)
  const int* src_row;  // (nx + 1) offsets into src
  const float* waveform;  // (nsrc, nsteps), rows in the sorted order
  int nrec;
  const int* rec;  // (nrec, 2) cell, field
  float* rec_out;
  int snap_field, snap_interval;
  float* snapshots;
};

enum { kOpCpml = 1, kOpPec = 2, kOpMur = 3 };

struct Strips {
  // low-side slot (= cell index) and profile index, high-side slot, for the
  // H rule (cells < n-1) or the E rule (cells > 0)
  int lo, lo_k, hi;
};
CEEP_D Strips strips(int i, int n, int t, bool h_rule) {
  Strips s{-1, -1, -1};
  const int m = h_rule ? min(t, n - 1) : min(t, n);
  if (i < m && (h_rule || i > 0)) {
    s.lo = i;
    s.lo_k = t - 1 - i;
  }
  const int k = i - (n - t);
  if (k >= 0 && k < m && (h_rule ? i < n - 1 : i > 0)) s.hi = k;
  return s;
}

// One CPML psi recurrence psi' = b psi + c diff / d, reading `q`; written to
// `out` when given (the owning cell), returned.
CEEP_D float psi_step(const float* q, float* out, float b, float c, float diff, float inv) {
  const float v = b * *q + c * diff * inv;
  if (out) *out = v;
  return v;
}

// The x-strip (t, ny) and y-strip (nx, t) psi slots of cell (i, j) in a
// psi array of the layout above; -1 when the cell is not on that side.
struct PsiSlots {
  long long xlo, xhi, ylo, yhi;
  int kxlo, kylo;
};
CEEP_D PsiSlots psi_slots(int i, int j, int nx, int ny, int t, bool h_rule) {
  PsiSlots s{-1, -1, -1, -1, 0, 0};
  const Strips sx = strips(i, nx, t, h_rule), sy = strips(j, ny, t, h_rule);
  if (sx.lo >= 0) { s.xlo = (long long)sx.lo * ny + j; s.kxlo = sx.lo_k; }
  if (sx.hi >= 0) s.xhi = (long long)(t + sx.hi) * ny + j;
  const long long yb = 2LL * t * ny;
  if (sy.lo >= 0) { s.ylo = yb + (long long)i * t + sy.lo; s.kylo = sy.lo_k; }
  if (sy.hi >= 0) s.yhi = yb + (long long)nx * t + (long long)i * t + sy.hi;
  return s;
}

// -- CPML H corrections of one cell (absorbing.py:332-451), given the E
// differences the cell's plain update used; psi is read from half r and, for
// the owning cell, written to half r^1.  Each returns the signed sum to add.
template <bool CPML>
CEEP_D float cpml_h_x(const Single2dParams& p, int r, int i, int c, float diff, bool own) {
  if (!CPML) return 0.f;
  const int t = p.t;
  const Strips sx = strips(i, p.nx, t, true);
  const float* bh = p.cpml + 2 * t;
  const float* chh = p.cpml + 3 * t;
  float acc = 0.f;
  if (sx.lo >= 0) {
    const long long q = (long long)sx.lo * p.ny + c;
    acc += p.dt_mu0 * psi_step(p.psi_h[r] + q, own ? p.psi_h[r ^ 1] + q : nullptr, bh[sx.lo_k], chh[sx.lo_k], diff,
                               p.inv_dx);
  }
  if (sx.hi >= 0) {
    const long long q = (long long)(t + sx.hi) * p.ny + c;
    acc += p.dt_mu0 * psi_step(p.psi_h[r] + q, own ? p.psi_h[r ^ 1] + q : nullptr, bh[sx.hi], chh[sx.hi], diff,
                               p.inv_dx);
  }
  return acc;
}

template <bool CPML>
CEEP_D float cpml_h_y(const Single2dParams& p, int r, int i, int c, float diff, bool own) {
  if (!CPML) return 0.f;
  const int t = p.t;
  const Strips sy = strips(c, p.ny, t, true);
  const float* bh = p.cpml + 6 * t;
  const float* chh = p.cpml + 7 * t;
  const long long yb = 2LL * t * p.ny;
  float acc = 0.f;
  if (sy.lo >= 0) {
    const long long q = yb + (long long)i * t + sy.lo;
    acc += p.dt_mu0 * psi_step(p.psi_h[r] + q, own ? p.psi_h[r ^ 1] + q : nullptr, bh[sy.lo_k], chh[sy.lo_k], diff,
                               p.inv_dy);
  }
  if (sy.hi >= 0) {
    const long long q = yb + (long long)p.nx * t + (long long)i * t + sy.hi;
    acc += p.dt_mu0 * psi_step(p.psi_h[r] + q, own ? p.psi_h[r ^ 1] + q : nullptr, bh[sy.hi], chh[sy.hi], diff,
                               p.inv_dy);
  }
  return acc;
}

// Plain + CPML H of one component at (i, c), everything loaded here: used
// for the row just below a segment, which the walk does not otherwise visit.
template <bool CPML>
CEEP_D float tmz_hy_at(const Single2dParams& p, int r, int i, int c) {
  const size_t k = (size_t)i * p.ny + c;
  const float* ez = p.f[0][r];
  const float dx = i + 1 < p.nx ? __ldg(ez + k + p.ny) - __ldg(ez + k) : 0.f;
  const float2 d = __ldg(p.ch + k);
  float v = __ldg(p.f[2][r] + k);
  if (i < p.nx - 1) v = d.x * v + (d.y * p.inv_dx) * dx;
  return v + cpml_h_x<CPML>(p, r, i, c, dx, false);
}

template <bool CPML>
CEEP_D float tez_hz_at(const Single2dParams& p, int r, int i, int c) {
  const size_t k = (size_t)i * p.ny + c;
  const float* ex = p.f[1][r];
  const float* ey = p.f[2][r];
  const float dex = c + 1 < p.ny ? __ldg(ex + k + 1) - __ldg(ex + k) : 0.f;
  const float dey = i + 1 < p.nx ? __ldg(ey + k + p.ny) - __ldg(ey + k) : 0.f;
  const float2 d = __ldg(p.ch + k);
  float v = __ldg(p.f[0][r] + k);
  if (i < p.nx - 1 && c < p.ny - 1) v = d.x * v + d.y * (dex * p.inv_dy - dey * p.inv_dx);
  return v - cpml_h_x<CPML>(p, r, i, c, dey, false) + cpml_h_y<CPML>(p, r, i, c, dex, false);
}

// CPML E corrections of the owning cell (absorbing.py:453-561), psi in place.
template <bool CPML>
CEEP_D float cpml_e_x(const Single2dParams& p, int i, int c, float diff) {
  if (!CPML) return 0.f;
  const int t = p.t;
  const Strips sx = strips(i, p.nx, t, false);
  float* q = p.psi_e;
  float acc = 0.f;
  if (sx.lo >= 0) {
    const long long o = (long long)sx.lo * p.ny + c;
    acc += p.dt_eps0 * psi_step(q + o, q + o, p.cpml[sx.lo_k], p.cpml[t + sx.lo_k], diff, p.inv_dx);
  }
  if (sx.hi >= 0) {
    const long long o = (long long)(t + sx.hi) * p.ny + c;
    acc += p.dt_eps0 * psi_step(q + o, q + o, p.cpml[sx.hi], p.cpml[t + sx.hi], diff, p.inv_dx);
  }
  return acc;
}

template <bool CPML>
CEEP_D float cpml_e_y(const Single2dParams& p, int i, int c, float diff) {
  if (!CPML) return 0.f;
  const int t = p.t;
  const Strips sy = strips(c, p.ny, t, false);
  const long long yb = 2LL * t * p.ny;
  float* q = p.psi_e;
  float acc = 0.f;
  if (sy.lo >= 0) {
    const long long o = yb + (long long)i * t + sy.lo;
    acc += p.dt_eps0 * psi_step(q + o, q + o, p.cpml[4 * t + sy.lo_k], p.cpml[5 * t + sy.lo_k], diff, p.inv_dy);
  }
  if (sy.hi >= 0) {
    const long long o = yb + (long long)p.nx * t + (long long)i * t + sy.hi;
    acc += p.dt_eps0 * psi_step(q + o, q + o, p.cpml[4 * t + sy.hi], p.cpml[5 * t + sy.hi], diff, p.inv_dy);
  }
  return acc;
}

// One step as a warp row-walk.  A warp covers columns j0-1 .. j0+30 (lane l
// at column j0-1+l) and owns j0 .. j0+30 (lanes 1..31); it walks its segment
// of rows upward.  At row i each lane forms the new H of its column;
// the E update of (i, c) then takes H(i, c-1) from the lane on its left by
// shuffle (lane 0 computes the column left of the strip for that purpose
// only and writes nothing), H(i-1, c) from the previous iteration's
// register, and E(i, c+1) / E(i+1, c) of the read half by shuffle and by
// carrying the next row.  The row below a segment is recomputed before the
// walk.  Fields and the H psi are ping-pong buffered, so those recomputes
// read values that no warp is writing; the E psi is touched by its own cell
// only.  No shared memory and no barriers: every field is read and written
// once and each coefficient pair read once per step.
// A block covers kBlockRows rows of a 31-column strip; its warps split them:
// 4 warps of 32 rows in the interior launch, 16 warps of 8 rows in the frame
// launch (few blocks, so shorter walks keep its duration down).
constexpr int kBlockRows = 128, kWarpsInterior = 4, kWarpsFrame = 16;
constexpr int kInteriorRows = 128;  // rows of one interior block (kWarpsInterior walks)

// Blocks of 31 columns x up to kBlockRows rows, split into an interior
// rectangle -- columns [col_lo, col_hi) over rows [row_lo, row_hi), whose
// cells and halo touch no CPML strip and no grid edge -- and the frame around
// it: a top band of rows [0, row_lo), a bottom band [row_hi, nx), both full
// width, and side blocks on the columns [0, col_lo) and [col_hi, ny) of the
// interior rows.  The interior launch runs the code without CPML (half the
// registers, twice the resident warps); the frame launch maps its linear
// block index onto the bands and sides.  Neither the rows nor the columns of
// the rectangle are rounded to whole blocks, so the frame holds little more
// than the strips themselves.
struct BlockMap {
  int gx;                       // column blocks of the bands
  int col_lo, col_hi, ny;       // interior columns [lo, hi); grid columns
  int row_lo, row_hi, nx;       // interior rows [lo, hi); grid rows
  int frame;                    // 0: interior launch (2D grid), 1: frame launch (1D grid)
};

__host__ __device__ inline int side_blocks(int cols) { return (cols + 30) / 31; }

// This block's first owned column j0, the end ce of the columns it owns (a
// side block may reach into the interior and owns only up to it), and its
// row range [rs, re).
CEEP_D void block_of(const BlockMap& m, int& j0, int& ce, int& rs, int& re) {
  if (!m.frame) {
    j0 = m.col_lo + blockIdx.x * 31;
    ce = m.col_hi;
    rs = m.row_lo + blockIdx.y * kInteriorRows;
    re = min(rs + kInteriorRows, m.row_hi);
    return;
  }
  ce = m.ny;
  int f = blockIdx.x;
  const int top = (m.row_lo + kBlockRows - 1) / kBlockRows * m.gx;
  if (f < top) {
    j0 = f % m.gx * 31;
    rs = f / m.gx * kBlockRows;
    re = min(rs + kBlockRows, m.row_lo);
    return;
  }
  f -= top;
  const int bottom = (m.nx - m.row_hi + kBlockRows - 1) / kBlockRows * m.gx;
  if (f < bottom) {
    j0 = f % m.gx * 31;
    rs = m.row_hi + f / m.gx * kBlockRows;
    re = min(rs + kBlockRows, m.nx);
    return;
  }
  f -= bottom;
  const int nl = side_blocks(m.col_lo), side = nl + side_blocks(m.ny - m.col_hi);
  rs = m.row_lo + f / side * kBlockRows;
  re = min(rs + kBlockRows, m.row_hi);
  const int q = f % side;
  if (q < nl) {
    j0 = q * 31;
    ce = m.col_lo;
  } else {
    j0 = m.col_hi + (q - nl) * 31;
  }
}

template <int MODE, bool CPML>
__global__ void __launch_bounds__(32 * kWarpsFrame) single2d_step_kernel(const Single2dParams p, int step, int r,
                                                                           const BlockMap bm) {
  const int w = r ^ 1;
  const int lane = threadIdx.x, nx = p.nx, ny = p.ny;
  int j0, ce, rs, re;
  block_of(bm, j0, ce, rs, re);
  const int c = j0 - 1 + lane;
  const int rows = (bm.frame ? kBlockRows : kInteriorRows) / blockDim.y;
  const int i0 = rs + threadIdx.y * rows;
  if (i0 >= re) return;  // whole warp
  const int i1 = min(i0 + rows, re);
  const bool live = c >= 0 && c < ny;
  const bool own = live && lane > 0 && c < ce;
  const int cl = live ? c : max(min(c, ny - 1), 0);  // a valid column for the non-live lanes' loads
  if (MODE == 0) {
    const float* ez_r = p.f[0][r];
    const float* hx_r = p.f[1][r];
    const float* hy_r = p.f[2][r];
    float hy_prev = 0.f;
    if (i0 > 0) hy_prev = tmz_hy_at<CPML>(p, r, i0 - 1, cl);
    // the read-half operands of the current row are loaded one iteration
    // ahead, before the current row's stores, so each warp keeps two rows of
    // loads in flight
    size_t k = (size_t)i0 * ny + cl;
    float ez_c = __ldg(ez_r + k);
    float ez_n = i0 + 1 < nx ? __ldg(ez_r + k + ny) : 0.f;
    float hx_c = __ldg(hx_r + k), hy_c = __ldg(hy_r + k);
    float2 d_c = __ldg(p.ch + k), e_c = __ldg(p.ce + k);
    for (int i = i0; i < i1; ++i, k += ny) {
      const bool more = i + 1 < i1;
      const float ez_nn = more && i + 2 < nx ? __ldg(ez_r + k + 2 * (size_t)ny) : 0.f;
      const float hx_n = more ? __ldg(hx_r + k + ny) : 0.f;
      const float hy_n = more ? __ldg(hy_r + k + ny) : 0.f;
      const float2 d_n = more ? __ldg(p.ch + k + ny) : make_float2(0.f, 0.f);
      const float2 e_n = more ? __ldg(p.ce + k + ny) : make_float2(0.f, 0.f);
      float ez_rt = __shfl_down_sync(0xffffffffu, ez_c, 1);
      if (lane == 31) ez_rt = c + 1 < ny ? __ldg(ez_r + k + 1) : 0.f;
      const float2 d = d_c;
      const float dy = c + 1 < ny ? ez_rt - ez_c : 0.f;
      const float dx = i + 1 < nx ? ez_n - ez_c : 0.f;
      float hx = hx_c, hy = hy_c;
      if (c < ny - 1) hx = d.x * hx - (d.y * p.inv_dy) * dy;
      if (i < nx - 1) hy = d.x * hy + (d.y * p.inv_dx) * dx;
      if (CPML) {
        hx -= cpml_h_y<CPML>(p, r, i, cl, dy, own);
        hy += cpml_h_x<CPML>(p, r, i, cl, dx, own);
      }
      const float hx_l = __shfl_up_sync(0xffffffffu, hx, 1);
      if (own) {
        p.f[1][w][k] = hx;
        p.f[2][w][k] = hy;
        // Ez on [1, nx) x [1, ny) (fdtd_2d.py:165-171)
        const float dhy = i > 0 ? hy - hy_prev : 0.f;
        const float dhx = c > 0 ? hx - hx_l : 0.f;
        const float2 kk = e_c;
        float e = ez_c;
        if (i > 0 && c > 0) e = kk.x * e + kk.y * (dhy * p.inv_dx - dhx * p.inv_dy);
        for (int s = __ldg(p.src_row + i); s < __ldg(p.src_row + i + 1); ++s)  // fdtd_2d.py:245-260
          if (__ldg(p.src + 3 * s + 1) == c && __ldg(p.src + 3 * s + 2) == 0)
            e += __ldg(p.waveform + (size_t)s * p.nsteps + step);
        for (int o = 0; o < p.n_ops; ++o) {
          if (CPML && p.ops[o] == kOpCpml) {
            e += cpml_e_x<CPML>(p, i, c, dhy);
            e -= cpml_e_y<CPML>(p, i, c, dhx);
          } else if (p.ops[o] == kOpPec && (i == 0 || i == nx - 1 || c == 0 || c == ny - 1)) {
            e = 0.f;  // absorbing.py:58-66
          }
        }
        p.f[0][w][k] = e;
      }
      hy_prev = hy;
      ez_c = ez_n;
      ez_n = ez_nn;
      hx_c = hx_n;
      hy_c = hy_n;
      d_c = d_n;
      e_c = e_n;
    }
  } else {
    const float* hz_r = p.f[0][r];
    const float* ex_r = p.f[1][r];
    const float* ey_r = p.f[2][r];
    float hz_prev = 0.f;
    if (i0 > 0) hz_prev = tez_hz_at<CPML>(p, r, i0 - 1, cl);
    size_t k = (size_t)i0 * ny + cl;
    float ey_c = __ldg(ey_r + k);
    float ey_n = i0 + 1 < nx ? __ldg(ey_r + k + ny) : 0.f;
    float ex_c = __ldg(ex_r + k), hz_c = __ldg(hz_r + k);
    float2 d_c = __ldg(p.ch + k), e_c = __ldg(p.ce + k);
    for (int i = i0; i < i1; ++i, k += ny) {
      const bool more = i + 1 < i1;
      const float ey_nn = more && i + 2 < nx ? __ldg(ey_r + k + 2 * (size_t)ny) : 0.f;
      const float ex_n = more ? __ldg(ex_r + k + ny) : 0.f;
      const float hz_n = more ? __ldg(hz_r + k + ny) : 0.f;
      const float2 d_n = more ? __ldg(p.ch + k + ny) : make_float2(0.f, 0.f);
      const float2 e_n = more ? __ldg(p.ce + k + ny) : make_float2(0.f, 0.f);
      float ex_rt = __shfl_down_sync(0xffffffffu, ex_c, 1);
      if (lane == 31) ex_rt = c + 1 < ny ? __ldg(ex_r + k + 1) : 0.f;
      const float2 d = d_c;
      const float dex = c + 1 < ny ? ex_rt - ex_c : 0.f;
      const float dey = i + 1 < nx ? ey_n - ey_c : 0.f;
      float hz = hz_c;
      if (i < nx - 1 && c < ny - 1) hz = d.x * hz + d.y * (dex * p.inv_dy - dey * p.inv_dx);
      if (CPML) {
        // x strips subtract, y strips add (absorbing.py:355-405)
        hz -= cpml_h_x<CPML>(p, r, i, cl, dey, own);
        hz += cpml_h_y<CPML>(p, r, i, cl, dex, own);
      }
      const float hz_l = __shfl_up_sync(0xffffffffu, hz, 1);
      if (own) {
        p.f[0][w][k] = hz;
        // Ex on c >= 1, Ey on i >= 1 (fdtd_2d.py:205-217)
        const float dy = c > 0 ? hz - hz_l : 0.f;
        const float dx = i > 0 ? hz - hz_prev : 0.f;
        const float2 kk = e_c;
        float vx = ex_c, vy = ey_c;
        if (c > 0) vx = kk.x * vx + (kk.y * p.inv_dy) * dy;
        if (i > 0) vy = kk.x * vy - (kk.y * p.inv_dx) * dx;
        for (int s = __ldg(p.src_row + i); s < __ldg(p.src_row + i + 1); ++s) {
          if (__ldg(p.src + 3 * s + 1) != c) continue;
          const int fld = __ldg(p.src + 3 * s + 2);
          const float wv = __ldg(p.waveform + (size_t)s * p.nsteps + step);
          if (fld == 1) vx += wv;
          else if (fld == 2) vy += wv;
        }
        for (int o = 0; o < p.n_ops; ++o) {
          if (CPML && p.ops[o] == kOpCpml) {
            // y strips on Ex first, then x strips on Ey (absorbing.py:467-511)
            vx += cpml_e_y<CPML>(p, i, c, dy);
            vy -= cpml_e_x<CPML>(p, i, c, dx);
          } else if (p.ops[o] == kOpPec) {
            if (i == 0 || i == nx - 1) vx = 0.f;  // absorbing.py:68-72
            if (c == 0 || c == ny - 1) vy = 0.f;
          }
        }
        p.f[1][w][k] = vx;
        p.f[2][w][k] = vy;
      }
      hz_prev = hz;
      ey_c = ey_n;
      ey_n = ey_nn;
      ex_c = ex_n;
      hz_c = hz_n;
      d_c = d_n;
      e_c = e_n;
    }
  }
}

// The TMz interior walk with two columns per lane: lane l holds columns
// c, c+1 with c = j0 - 2 + 2l even, so every field row is read and written
// as float2 and every coefficient pair as float4 (twice the bytes in flight
// per warp of the one-column walk, half the load instructions).  Strips are
// 62 columns wide (lanes 1..31 own them; lane 0 forms the H of column j0-1
// for its neighbour's E update, and writes nothing).  Needs an even ny (the
// float2 rows stay aligned) and strip starts j0 on even columns; the
// cells it owns and their halo lie in the CPML- and edge-free interior, so
// the region tests of the general walk fold away.  Same arithmetic, in the
// same order, as the one-column walk.
__global__ void __launch_bounds__(32 * kWarpsInterior) single2d_tmz_pair_kernel(const Single2dParams p, int step,
                                                                                 int r, int col_lo, int row_lo,
                                                                                 int row_hi) {
  const int w = r ^ 1;
  const int lane = threadIdx.x, nx = p.nx, ny = p.ny;
  const int j0 = col_lo + 62 * blockIdx.x;
  const int c = j0 - 2 + 2 * lane;
  constexpr int rows = kInteriorRows / kWarpsInterior;
  const int i0 = row_lo + blockIdx.y * kInteriorRows + threadIdx.y * rows;
  if (i0 >= row_hi) return;  // whole warp
  const int i1 = min(i0 + rows, row_hi);
  const bool own = lane > 0;
  const float* ez_r = p.f[0][r];
  const float2* ez2 = reinterpret_cast<const float2*>(ez_r);
  const float2* hx2 = reinterpret_cast<const float2*>(p.f[1][r]);
  const float2* hy2 = reinterpret_cast<const float2*>(p.f[2][r]);
  const float4* ch4 = reinterpret_cast<const float4*>(p.ch);  // (da, db) of c, then of c+1
  const float4* ce4 = reinterpret_cast<const float4*>(p.ce);  // (ca, cb) of c, then of c+1
  float2* ez_w = reinterpret_cast<float2*>(p.f[0][w]);
  float2* hx_w = reinterpret_cast<float2*>(p.f[1][w]);
  float2* hy_w = reinterpret_cast<float2*>(p.f[2][w]);
  const size_t row2 = (size_t)ny / 2;
  float2 hy_prev = make_float2(tmz_hy_at<false>(p, r, i0 - 1, c), tmz_hy_at<false>(p, r, i0 - 1, c + 1));
  size_t k = ((size_t)i0 * ny + c) / 2;
  float2 ez_c = __ldg(ez2 + k);
  float2 ez_n = __ldg(ez2 + k + row2);
  float2 hx_c = __ldg(hx2 + k), hy_c = __ldg(hy2 + k);
  float4 d_c = __ldg(ch4 + k), e_c = __ldg(ce4 + k);
  const float z2 = 0.f;
  for (int i = i0; i < i1; ++i, k += row2) {
    const bool more = i + 1 < i1;
    const float2 ez_nn = more && i + 2 < nx ? __ldg(ez2 + k + 2 * row2) : make_float2(z2, z2);
    const float2 hx_n = more ? __ldg(hx2 + k + row2) : make_float2(z2, z2);
    const float2 hy_n = more ? __ldg(hy2 + k + row2) : make_float2(z2, z2);
    const float4 d_n = more ? __ldg(ch4 + k + row2) : make_float4(z2, z2, z2, z2);
    const float4 e_n = more ? __ldg(ce4 + k + row2) : make_float4(z2, z2, z2, z2);
    float ez_rt = __shfl_down_sync(0xffffffffu, ez_c.x, 1);
    if (lane == 31) ez_rt = __ldg(ez_r + (size_t)i * ny + c + 2);
    float2 hx, hy;
    hx.x = d_c.x * hx_c.x - (d_c.y * p.inv_dy) * (ez_c.y - ez_c.x);
    hx.y = d_c.z * hx_c.y - (d_c.w * p.inv_dy) * (ez_rt - ez_c.y);
    hy.x = d_c.x * hy_c.x + (d_c.y * p.inv_dx) * (ez_n.x - ez_c.x);
    hy.y = d_c.z * hy_c.y + (d_c.w * p.inv_dx) * (ez_n.y - ez_c.y);
    const float hx_l = __shfl_up_sync(0xffffffffu, hx.y, 1);
    if (own) {
      hx_w[k] = hx;
      hy_w[k] = hy;
      float2 e;
      e.x = e_c.x * ez_c.x + e_c.y * ((hy.x - hy_prev.x) * p.inv_dx - (hx.x - hx_l) * p.inv_dy);
      e.y = e_c.z * ez_c.y + e_c.w * ((hy.y - hy_prev.y) * p.inv_dx - (hx.y - hx.x) * p.inv_dy);
      for (int s = __ldg(p.src_row + i); s < __ldg(p.src_row + i + 1); ++s) {  // fdtd_2d.py:245-260
        if (__ldg(p.src + 3 * s + 2) != 0) continue;
        const int sc = __ldg(p.src + 3 * s + 1);
        if (sc == c) e.x += __ldg(p.waveform + (size_t)s * p.nsteps + step);
        else if (sc == c + 1) e.y += __ldg(p.waveform + (size_t)s * p.nsteps + step);
      }
      ez_w[k] = e;
    }
    hy_prev = hy;
    ez_c = ez_n;
    ez_n = ez_nn;
    hx_c = hx_n;
    hy_c = hy_n;
    d_c = d_n;
    e_c = e_n;
  }
}

// The TEz interior walk with two columns per lane, as the TMz one above:
// Hz from the Ex / Ey differences, then Ex and Ey from Hz of the left lane
// and of the row below.  Same arithmetic, in the same order, as the
// one-column walk.
__global__ void __launch_bounds__(32 * kWarpsInterior) single2d_tez_pair_kernel(const Single2dParams p, int step,
                                                                                 int r, int col_lo, int row_lo,
                                                                                 int row_hi) {
  const int w = r ^ 1;
  const int lane = threadIdx.x, nx = p.nx, ny = p.ny;
  const int j0 = col_lo + 62 * blockIdx.x;
  const int c = j0 - 2 + 2 * lane;
  constexpr int rows = kInteriorRows / kWarpsInterior;
  const int i0 = row_lo + blockIdx.y * kInteriorRows + threadIdx.y * rows;
  if (i0 >= row_hi) return;  // whole warp
  const int i1 = min(i0 + rows, row_hi);
  const bool own = lane > 0;
  const float* ex_r = p.f[1][r];
  const float2* hz2 = reinterpret_cast<const float2*>(p.f[0][r]);
  const float2* ex2 = reinterpret_cast<const float2*>(ex_r);
  const float2* ey2 = reinterpret_cast<const float2*>(p.f[2][r]);
  const float4* ch4 = reinterpret_cast<const float4*>(p.ch);  // (da, db) of c, then of c+1
  const float4* ce4 = reinterpret_cast<const float4*>(p.ce);  // (ca, cb) of c, then of c+1
  float2* hz_w = reinterpret_cast<float2*>(p.f[0][w]);
  float2* ex_w = reinterpret_cast<float2*>(p.f[1][w]);
  float2* ey_w = reinterpret_cast<float2*>(p.f[2][w]);
  const size_t row2 = (size_t)ny / 2;
  float2 hz_prev = make_float2(tez_hz_at<false>(p, r, i0 - 1, c), tez_hz_at<false>(p, r, i0 - 1, c + 1));
  size_t k = ((size_t)i0 * ny + c) / 2;
  float2 ey_c = __ldg(ey2 + k);
  float2 ey_n = __ldg(ey2 + k + row2);
  float2 ex_c = __ldg(ex2 + k), hz_c = __ldg(hz2 + k);
  float4 d_c = __ldg(ch4 + k), e_c = __ldg(ce4 + k);
  const float z2 = 0.f;
  for (int i = i0; i < i1; ++i, k += row2) {
    const bool more = i + 1 < i1;
    const float2 ey_nn = more && i + 2 < nx ? __ldg(ey2 + k + 2 * row2) : make_float2(z2, z2);
    const float2 ex_n = more ? __ldg(ex2 + k + row2) : make_float2(z2, z2);
    const float2 hz_n = more ? __ldg(hz2 + k + row2) : make_float2(z2, z2);
    const float4 d_n = more ? __ldg(ch4 + k + row2) : make_float4(z2, z2, z2, z2);
    const float4 e_n = more ? __ldg(ce4 + k + row2) : make_float4(z2, z2, z2, z2);
    float ex_rt = __shfl_down_sync(0xffffffffu, ex_c.x, 1);
    if (lane == 31) ex_rt = __ldg(ex_r + (size_t)i * ny + c + 2);
    float2 hz;
    hz.x = d_c.x * hz_c.x + d_c.y * ((ex_c.y - ex_c.x) * p.inv_dy - (ey_n.x - ey_c.x) * p.inv_dx);
    hz.y = d_c.z * hz_c.y + d_c.w * ((ex_rt - ex_c.y) * p.inv_dy - (ey_n.y - ey_c.y) * p.inv_dx);
    const float hz_l = __shfl_up_sync(0xffffffffu, hz.y, 1);
    if (own) {
      hz_w[k] = hz;
      float2 vx, vy;
      vx.x = e_c.x * ex_c.x + (e_c.y * p.inv_dy) * (hz.x - hz_l);
      vx.y = e_c.z * ex_c.y + (e_c.w * p.inv_dy) * (hz.y - hz.x);
      vy.x = e_c.x * ey_c.x - (e_c.y * p.inv_dx) * (hz.x - hz_prev.x);
      vy.y = e_c.z * ey_c.y - (e_c.w * p.inv_dx) * (hz.y - hz_prev.y);
      for (int s = __ldg(p.src_row + i); s < __ldg(p.src_row + i + 1); ++s) {  // fdtd_2d.py:245-260
        const int sc = __ldg(p.src + 3 * s + 1);
        if (sc != c && sc != c + 1) continue;
        const int fld = __ldg(p.src + 3 * s + 2);
        const float wv = __ldg(p.waveform + (size_t)s * p.nsteps + step);
        float2& v = fld == 1 ? vx : vy;
        if (fld == 1 || fld == 2) {
          if (sc == c) v.x += wv;
          else v.y += wv;
        }
      }
      ex_w[k] = vx;
      ey_w[k] = vy;
    }
    hz_prev = hz;
    ey_c = ey_n;
    ey_n = ey_nn;
    ex_c = ex_n;
    hz_c = hz_n;
    d_c = d_n;
    e_c = e_n;
  }
}

// TEz Hz sources, in list order (fdtd_2d.py:253-254).
__global__ void single2d_src_h_kernel(const Single2dParams p, int step, int cur) {
  if (threadIdx.x != 0) return;
  for (int s = 0; s < p.nsrc; ++s)
    if (p.src[3 * s + 2] == 0)
      p.f[0][cur][(size_t)p.src[3 * s] * p.ny + p.src[3 * s + 1]] += p.waveform[(size_t)s * p.nsteps + step];
}

// First-order Mur on the edges of field 0 (absorbing.py:126-166).  prev holds
// the previous step's lines next to the edges (x0, xn: ny each; y0, yn: nx
// each); this step's lines go to the other half of the pair.
__global__ void single2d_mur_kernel(const Single2dParams p, int step, int cur) {
  const int nx = p.nx, ny = p.ny;
  float* e = p.f[0][cur];
  const int len = 2 * ny + 2 * nx;
  const float* prev = p.mur_prev + (size_t)(step & 1) * len;
  float* next = p.mur_prev + (size_t)((step + 1) & 1) * len;
  for (int j = threadIdx.x; j < ny; j += blockDim.x) {
    next[j] = e[(size_t)ny + j];
    next[ny + j] = e[(size_t)(nx - 2) * ny + j];
  }
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    next[2 * ny + i] = e[(size_t)i * ny + 1];
    next[2 * ny + nx + i] = e[(size_t)i * ny + ny - 2];
  }
  __syncthreads();
  for (int j = threadIdx.x; j < ny; j += blockDim.x) {
    const float a0 = e[j], a1 = e[(size_t)ny + j];
    const float b0 = e[(size_t)(nx - 1) * ny + j], b1 = e[(size_t)(nx - 2) * ny + j];
    e[j] = prev[j] + p.mur_kx * (a1 - a0);
    e[(size_t)(nx - 1) * ny + j] = prev[ny + j] + p.mur_kx * (b1 - b0);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < nx; i += blockDim.x) {
    float* r = e + (size_t)i * ny;
    const float a0 = r[0], a1 = r[1], b0 = r[ny - 1], b1 = r[ny - 2];
    r[0] = prev[2 * ny + i] + p.mur_ky * (a1 - a0);
    r[ny - 1] = prev[2 * ny + nx + i] + p.mur_ky * (b1 - b0);
  }
}

__global__ void single2d_record_kernel(const Single2dParams p, int step, int cur) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.nrec) return;
  p.rec_out[(size_t)r * p.nsteps + step] = p.f[p.rec[2 * r + 1]][cur][p.rec[2 * r]];
}

// The interior rectangle for a walk of `width`-column strips (31, or 62 for
// the two-column walk, whose strips start on even columns): owned columns
// and rows with their halo (the column and row on each side) inside
// [e, n-e) with e = max(t, 1), i.e. clear of the CPML strips and the edges.
BlockMap block_map(const Single2dParams& p, int width) {
  BlockMap m;
  m.gx = (p.ny + 30) / 31;
  m.nx = p.nx;
  m.ny = p.ny;
  const int e = p.t > 1 ? p.t : 1;
  m.col_lo = e + 1;
  if (width == 62) m.col_lo += m.col_lo & 1;
  const int strips_n = p.ny - e - m.col_lo >= 0 ? (p.ny - e - m.col_lo) / width : 0;
  m.col_hi = m.col_lo + strips_n * width;
  m.row_lo = e + 1;
  m.row_hi = p.nx - e;
  if (strips_n <= 0 || m.row_hi <= m.row_lo) m.col_lo = m.col_hi = m.row_lo = m.row_hi = 0;
  m.frame = 0;
  return m;
}

// The frame launch (few blocks, latency-bound walks) runs on a second stream
// beside the interior launch; both read only the read half and write
// disjoint cells of the write half.
template <int MODE, bool CPML>
static cudaError_t step_t(const Single2dParams& p, int step, int r, cudaStream_t s, cudaStream_t s2,
                          cudaEvent_t fork, cudaEvent_t join) {
  // an even ny: the interior runs the two-column walk (62-column strips
  // starting on an even column)
  const bool pair = p.ny % 2 == 0;
  const int width = pair ? 62 : 31;
  BlockMap m = block_map(p, width);
  const int ibx = (m.col_hi - m.col_lo) / width;                            // interior strips
  const int iby = (m.row_hi - m.row_lo + kInteriorRows - 1) / kInteriorRows;   // interior block rows
  const int interior = ibx * iby;
  const int fby = (m.row_hi - m.row_lo + kBlockRows - 1) / kBlockRows;      // frame side block rows
  const int rest = (m.row_lo + kBlockRows - 1) / kBlockRows * m.gx +
                   (m.nx - m.row_hi + kBlockRows - 1) / kBlockRows * m.gx +
                   fby * (side_blocks(m.col_lo) + side_blocks(m.ny - m.col_hi));
  const bool two = interior > 0 && rest > 0;
  cudaError_t e;
  if (two) {
    if ((e = cudaEventRecord(fork, s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s2, fork, 0)) != cudaSuccess) return e;
  }
  if (rest > 0) {
    BlockMap f = m;
    f.frame = 1;
    single2d_step_kernel<MODE, CPML><<<rest, dim3(32, kWarpsFrame), 0, two ? s2 : s>>>(p, step, r, f);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (interior > 0) {
    if (pair && MODE == 0)
      single2d_tmz_pair_kernel<<<dim3(ibx, iby), dim3(32, kWarpsInterior), 0, s>>>(p, step, r, m.col_lo, m.row_lo,
                                                                                    m.row_hi);
    else if (pair)
      single2d_tez_pair_kernel<<<dim3(ibx, iby), dim3(32, kWarpsInterior), 0, s>>>(p, step, r, m.col_lo, m.row_lo,
                                                                                    m.row_hi);
    else
      single2d_step_kernel<MODE, false><<<dim3(ibx, iby), dim3(32, kWarpsInterior), 0, s>>>(p, step, r, m);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
  }
  if (two) {
    if ((e = cudaEventRecord(join, s2)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s, join, 0)) != cudaSuccess) return e;
  }
  return cudaSuccess;
}

}  // namespace ceep

struct ceep2s_plan {
  ceep::Single2dParams p;
  bool hz_src = false, mur = false, cpml = false;
  int cur = 0;  // the half of every ping-pong array holding the current state
  cudaStream_t side = nullptr;  // the frame launch's stream
  cudaEvent_t fork = nullptr, join = nullptr;
  std::map<std::tuple<int64_t, int64_t, int>, cudaGraphExec_t> graphs;
  std::set<std::tuple<int64_t, int64_t, int>> seen;  // step ranges run once without a graph
};

static int run_steps2s(const ceep2s_plan* pl, int64_t step0, int64_t nsteps, int cur, cudaStream_t s) {
  const ceep::Single2dParams& p = pl->p;
  for (int64_t k = 0; k < nsteps; ++k, cur ^= 1) {
    const int step = (int)(step0 + k);
    cudaError_t e;
    if (p.mode == 0)
      e = pl->cpml ? ceep::step_t<0, true>(p, step, cur, s, pl->side, pl->fork, pl->join)
                   : ceep::step_t<0, false>(p, step, cur, s, pl->side, pl->fork, pl->join);
    else
      e = pl->cpml ? ceep::step_t<1, true>(p, step, cur, s, pl->side, pl->fork, pl->join)
                   : ceep::step_t<1, false>(p, step, cur, s, pl->side, pl->fork, pl->join);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "single2d step launch");
    const int nw = cur ^ 1;
    if (pl->hz_src) ceep::single2d_src_h_kernel<<<1, 32, 0, s>>>(p, step, nw);
    if (pl->mur) ceep::single2d_mur_kernel<<<1, 1024, 0, s>>>(p, step, nw);
    if (p.nrec) ceep::single2d_record_kernel<<<(p.nrec + 255) / 256, 256, 0, s>>>(p, step, nw);
    e = cudaGetLastError();
    if (e != cudaSuccess) return ceep::cuda_fail(e, "single2d epilogue launch");
    if (p.snapshots && step % p.snap_interval == 0) {
      const size_t n = (size_t)p.nx * p.ny;
      e = cudaMemcpyAsync(p.snapshots + (size_t)(step / p.snap_interval) * n, p.f[p.snap_field][nw],
                          n * sizeof(float), cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return ceep::cuda_fail(e, "single2d snapshot copy");
    }
  }
  return CEEP_OK;
}

extern "C" int64_t ceep2s_desc_size(void) { return (int64_t)sizeof(ceep2s_desc); }

extern "C" int ceep2s_plan_create(const ceep2s_desc* d, ceep2s_plan** out) {
  using ceep::fail;
  if (!d || !out) return fail(CEEP_ERR_INVALID, "ceep2s_plan_create: null argument");
  *out = nullptr;
  if (d->nx < 3 || d->ny < 3) return fail(CEEP_ERR_INVALID, "grid %dx%d: at least 3x3", d->nx, d->ny);
  if (d->mode != 0 && d->mode != 1) return fail(CEEP_ERR_INVALID, "mode %d (0 TMz, 1 TEz)", d->mode);
  if (d->nsteps < 1) return fail(CEEP_ERR_INVALID, "nsteps %d", d->nsteps);
  for (int k = 0; k < 2; ++k)
    if (!d->f0[k] || !d->f1[k] || !d->f2[k]) return fail(CEEP_ERR_INVALID, "null field buffer");
  if (!d->coef_e || !d->coef_h) return fail(CEEP_ERR_INVALID, "null coefficient buffer");
  if (d->n_ops < 0 || d->n_ops > 4) return fail(CEEP_ERR_INVALID, "n_ops %d (at most 4)", d->n_ops);
  bool cpml = false, mur = false;
  for (int o = 0; o < d->n_ops; ++o) {
    const int op = d->ops[o];
    if (op != ceep::kOpCpml && op != ceep::kOpPec && op != ceep::kOpMur)
      return fail(CEEP_ERR_INVALID, "boundary op %d", op);
    if (op == ceep::kOpCpml) {
      if (cpml) return fail(CEEP_ERR_UNSUPPORTED, "one CPML per plan");
      cpml = true;
    }
    if (op == ceep::kOpMur) {
      if (o != d->n_ops - 1) return fail(CEEP_ERR_UNSUPPORTED, "Mur must be the last boundary");
      mur = true;
    }
  }
  if (cpml && (d->cpml_t < 1 || !d->cpml || !d->psi_e || !d->psi_h[0] || !d->psi_h[1]))
    return fail(CEEP_ERR_INVALID, "CPML: thickness/buffers");
  if (mur && !d->mur_prev) return fail(CEEP_ERR_INVALID, "Mur: null state buffer");
  if (d->nsrc < 0 || (d->nsrc && (!d->src || !d->src_row || !d->waveform)))
    return fail(CEEP_ERR_INVALID, "sources");
  if (d->nrec < 0 || (d->nrec && (!d->rec || !d->rec_out))) return fail(CEEP_ERR_INVALID, "record cells");
  if (d->snapshots && (d->snap_interval < 1 || d->snap_field < 0 || d->snap_field > 2))
    return fail(CEEP_ERR_INVALID, "snapshots: interval %d field %d", d->snap_interval, d->snap_field);
  const bool hz_src = d->mode == 1 && d->hz_sources != 0 && d->nsrc > 0;
  ceep2s_plan* pl = new (std::nothrow) ceep2s_plan();
  if (!pl) return fail(CEEP_ERR_INVALID, "host allocation failed");
  ceep::Single2dParams& p = pl->p;
  p.nx = d->nx; p.ny = d->ny; p.mode = d->mode; p.nsteps = d->nsteps;
  p.inv_dx = d->inv_dx; p.inv_dy = d->inv_dy; p.dt_mu0 = d->dt_mu0; p.dt_eps0 = d->dt_eps0;
  p.mur_kx = d->mur_kx; p.mur_ky = d->mur_ky;
  for (int k = 0; k < 2; ++k) {
    p.f[0][k] = d->f0[k];
    p.f[1][k] = d->f1[k];
    p.f[2][k] = d->f2[k];
    p.psi_h[k] = d->psi_h[k];
  }
  p.ce = reinterpret_cast<const float2*>(d->coef_e);
  p.ch = reinterpret_cast<const float2*>(d->coef_h);
  p.n_ops = d->n_ops;
  for (int o = 0; o < 4; ++o) p.ops[o] = o < d->n_ops ? d->ops[o] : 0;
  p.t = cpml ? d->cpml_t : 0;
  p.cpml = d->cpml; p.psi_e = d->psi_e; p.mur_prev = d->mur_prev;
  p.nsrc = d->nsrc; p.src = d->src; p.src_row = d->src_row; p.waveform = d->waveform;
  p.nrec = d->nrec; p.rec = d->rec; p.rec_out = d->rec_out;
  p.snap_field = d->snap_field; p.snap_interval = d->snap_interval > 0 ? d->snap_interval : 1;
  p.snapshots = d->snapshots;
  pl->cpml = cpml;
  pl->mur = mur;
  pl->hz_src = hz_src;
  cudaError_t e = cudaStreamCreateWithFlags(&pl->side, cudaStreamNonBlocking);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pl->fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pl->join, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    if (pl->fork) cudaEventDestroy(pl->fork);
    if (pl->side) cudaStreamDestroy(pl->side);
    delete pl;
    return ceep::cuda_fail(e, "ceep2s_plan_create stream/events");
  }
  *out = pl;
  return CEEP_OK;
}

extern "C" int ceep2s_plan_run(ceep2s_plan* pl, int64_t step0, int64_t nsteps, void* stream, int use_graph) {
  using ceep::fail;
  if (!pl) return fail(CEEP_ERR_INVALID, "null plan");
  if (step0 < 0 || nsteps < 0 || step0 + nsteps > pl->p.nsteps)
    return fail(CEEP_ERR_INVALID, "steps [%lld, %lld) outside [0, %d)", (long long)step0,
                (long long)(step0 + nsteps), pl->p.nsteps);
  if (nsteps == 0) return CEEP_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int cur = pl->cur;
  const int cur_after = cur ^ (int)(nsteps & 1);
  if (!use_graph || s == nullptr) {
    const int rc = run_steps2s(pl, step0, nsteps, cur, s);
    if (rc == CEEP_OK) pl->cur = cur_after;
    return rc;
  }
  auto key = std::make_tuple(step0, nsteps, cur);
  auto it = pl->graphs.find(key);
  if (it == pl->graphs.end() && pl->seen.insert(key).second) {
    // first request of this range: launch directly (a one-off run does not
    // pay for a capture); a second request captures it
    const int rc = run_steps2s(pl, step0, nsteps, cur, s);
    if (rc == CEEP_OK) pl->cur = cur_after;
    return rc;
  }
  if (it == pl->graphs.end()) {
    cudaGraph_t g;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "cudaStreamBeginCapture");
    int rc = run_steps2s(pl, step0, nsteps, cur, s);
    e = cudaStreamEndCapture(s, &g);
    if (rc != CEEP_OK) {
      if (e == cudaSuccess) cudaGraphDestroy(g);
      return rc;
    }
    if (e != cudaSuccess) return ceep::cuda_fail(e, "cudaStreamEndCapture");
    cudaGraphExec_t ex;
    e = cudaGraphInstantiate(&ex, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "cudaGraphInstantiate");
    it = pl->graphs.emplace(key, ex).first;
  }
  cudaError_t e = cudaGraphLaunch(it->second, s);
  if (e != cudaSuccess) return ceep::cuda_fail(e, "cudaGraphLaunch");
  pl->cur = cur_after;
  return CEEP_OK;
}

extern "C" int ceep2s_plan_current_buffer(const ceep2s_plan* pl) { return pl ? pl->cur : -1; }

extern "C" int ceep2s_plan_set_current_buffer(ceep2s_plan* pl, int cur) {
  if (!pl || (cur != 0 && cur != 1)) return ceep::fail(CEEP_ERR_INVALID, "bad plan or buffer index");
  pl->cur = cur;
  return CEEP_OK;
}

extern "C" int ceep2s_plan_destroy(ceep2s_plan* pl) {
  if (!pl) return CEEP_OK;
  for (auto& kv : pl->graphs) cudaGraphExecDestroy(kv.second);
  if (pl->side) cudaStreamSynchronize(pl->side);
  if (pl->join) cudaEventDestroy(pl->join);
  if (pl->fork) cudaEventDestroy(pl->fork);
  if (pl->side) cudaStreamDestroy(pl->side);
  delete pl;
  return CEEP_OK;
}

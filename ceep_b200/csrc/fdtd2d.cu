// Fused 2D TMz batched FDTD step for sm_100a.
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
// Layout: every field is (y, x, tx) with tx innermost and padded to a
// multiple of 4, so one float4 holds four transmit events of one cell and a
// warp reads 32 consecutive float4 (512 B) per field and row.  All cell
// coefficients (ca, cb, CPML, ADE) are loaded once per cell and serve every
// transmit event in the float4s of that cell.
//
// Fusion: E(x,y) needs H^{n+1/2} at (x-1,y) and (x,y-1).  Each thread walks
// a column segment upward in y, carrying Hx(x,y-1) and Ez(x,y+1) in
// registers, and recomputes Hy(x-1,y) from Ez (two extra FMAs per TX) rather
// than waiting for its neighbour.  Fields and the H-psi arrays are ping-pong
// buffered (read [p], write [p^1]) so these halo recomputes never race with
// the owner's write; the E-psi and ADE arrays are touched only by their
// owner and are updated in place.
//
// Per cell-step DRAM traffic: Ez, Hx, Hy read and written once (24 B per TX)
// plus 8 B of (ca, cb) per cell shared by all TX; strip cells add their psi.
#include "common.cuh"
#include "fdtd2d.cuh"

namespace ceep {

// ------------------------------------------------------------------------
// Per-cell updates.  `GEN` = false for blocks that lie entirely in the
// interior of every region (no strips, no edges): the predicates fold away.
// ------------------------------------------------------------------------

// Hx^{n+1/2}(x, y) from Ez(x,y), Ez(x,y+1)
template <bool GEN>
CEEP_D float4 hx_new(const Fdtd2dParams& p, int x, int y, int par, int l, float4 hx, float4 ez_c,
                     float4 ez_up, bool write_psi) {
  const int n = p.n;
  if (!GEN) return fma4(-p.db_dx, ez_up - ez_c, hx);
  if (y >= p.ny - 1) return hx;  // never updated
  float4 d = ez_up - ez_c;
  if (x >= n && x < p.nx - n && y >= n) hx = fma4(-p.db_dx, d, hx);
  int sy = -1, ci = 0;
  if (y < n) { sy = y; ci = y; }
  else if (y >= p.ny - n) { sy = n + (y - (p.ny - n)); ci = p.ny - 1 - y; }
  if (sy >= 0) {
    size_t idx = ((size_t)sy * p.nx + x) * p.lanes + l;
    float4 psi = ld4(p.psi_hx[par] + idx);
    psi = p.cpml_b[ci] * psi + p.cpml_c[ci] * (d * f4(p.inv_dx));
    if (write_psi) st4(p.psi_hx[par ^ 1] + idx, psi);
    hx = fma4(-p.db, psi, hx);
  }
  return hx;
}

// Hy^{n+1/2}(x, y) from Ez(x,y), Ez(x+1,y)
template <bool GEN>
CEEP_D float4 hy_new(const Fdtd2dParams& p, int x, int y, int par, int l, float4 hy, float4 ez_c,
                     float4 ez_r, bool write_psi) {
  const int n = p.n;
  if (!GEN) return fma4(p.db_dx, ez_r - ez_c, hy);
  if (x >= p.nx - 1) return hy;  // never updated
  float4 d = ez_r - ez_c;
  if (x >= n && y >= n && y < p.ny - n) hy = fma4(p.db_dx, d, hy);
  int sx = -1, ci = 0;
  if (x < n) { sx = x; ci = x; }
  else if (x >= p.nx - n) { sx = n + (x - (p.nx - n)); ci = p.nx - 1 - x; }
  if (sx >= 0) {
    size_t idx = ((size_t)y * (2 * n) + sx) * p.lanes + l;
    float4 psi = ld4(p.psi_hy[par] + idx);
    psi = p.cpml_b[ci] * psi + p.cpml_c[ci] * (d * f4(p.inv_dx));
    if (write_psi) st4(p.psi_hy[par ^ 1] + idx, psi);
    hy = fma4(p.db, psi, hy);
  }
  return hy;
}

// ADE on the interior E update (dispersive.py:364-404, fdtd_2d.py:163-178):
//   E  = ca*E_old + cb*curl - cb*sum(gamma_p J_p)
//   Debye   J = k1 J + k2 (E - E_old)/dt
//   Lorentz J' = k1 J + k3 J_prev + k2 (E - E_old)/dt ; J_prev = J ; J = J'
template <int ND, int NL>
CEEP_D float4 ade_update(const Fdtd2dParams& p, size_t cell, int l, float4 e_new, float4 e_old, float cb) {
  constexpr int NP = ND + NL;
  float4 J[NP > 0 ? NP : 1];
  float4 k[NP > 0 ? NP : 1];
  const size_t plane = (size_t)p.nx * p.ny;
  float4 sum = f4(0.f);
#pragma unroll
  for (int q = 0; q < NP; ++q) {
    k[q] = __ldg(reinterpret_cast<const float4*>(p.ade_coef) + q * plane + cell);
    J[q] = p.j[(q * plane + cell) * p.lanes + l];
    sum = (q < ND) ? fma4(k[q].z, J[q], sum) : sum + J[q];
  }
  e_new = e_new - cb * sum;
  float4 dedt = (e_new - e_old) / p.dt;
#pragma unroll
  for (int q = 0; q < NP; ++q) {
    float4* jp = p.j + (q * plane + cell) * p.lanes + l;
    if (q < ND) {
      *jp = k[q].x * J[q] + k[q].y * dedt;
    } else {
      float4* jq = p.j_prev + ((q - ND) * plane + cell) * p.lanes + l;
      float4 jm = *jq;
      *jp = k[q].x * J[q] + k[q].z * jm + k[q].y * dedt;
      *jq = J[q];
    }
  }
  return e_new;
}

template <int L, bool GEN, int ND, int NL>
CEEP_D void column_segment(const Fdtd2dParams& p, int x, int l, int y0, int y1, int step, int par) {
  const int nx = p.nx, ny = p.ny, n = p.n;
  const size_t rowstride = (size_t)nx * p.lanes;
  const float4* ez = p.ez[par];
  const float4* hxo = p.hx[par];
  const float4* hyo = p.hy[par];
  float4* ezw = p.ez[par ^ 1];
  float4* hxw = p.hx[par ^ 1];
  float4* hyw = p.hy[par ^ 1];
  const size_t col = (size_t)x * p.lanes + l;

  // prologue: Ez(x, y0) and Hx^{n+1/2}(x, y0-1)
  float4 ez_c = ld4(ez + (size_t)y0 * rowstride + col);
  float4 hx_prev = f4(0.f);
  if (y0 >= 1) {
    float4 ez_dn = ld4(ez + (size_t)(y0 - 1) * rowstride + col);
    hx_prev = hx_new<GEN>(p, x, y0 - 1, par, l, ld4(hxo + (size_t)(y0 - 1) * rowstride + col), ez_dn, ez_c,
                          false);
  }

  for (int y = y0; y < y1; ++y) {
    const size_t at = (size_t)y * rowstride + col;
    const float4 ez_up = (!GEN || y + 1 < ny) ? ld4(ez + at + rowstride) : f4(0.f);
    const float4 ez_r = (!GEN || x + 1 < nx) ? ld4(ez + at + p.lanes) : f4(0.f);
    const float4 ez_l = (!GEN || x >= 1) ? ld4(ez + at - p.lanes) : f4(0.f);

    // H phase (this cell, plus the recomputed Hy of the left neighbour)
    const float4 hxn = hx_new<GEN>(p, x, y, par, l, ld4(hxo + at), ez_c, ez_up, true);
    const float4 hyn = hy_new<GEN>(p, x, y, par, l, ld4(hyo + at), ez_c, ez_r, true);
    float4 hyl = f4(0.f);
    if (!GEN || x >= 1) hyl = hy_new<GEN>(p, x - 1, y, par, l, ld4(hyo + at - p.lanes), ez_l, ez_c, false);
    st4(hxw + at, hxn);
    st4(hyw + at, hyn);

    // E phase
    const size_t cell = (size_t)y * nx + x;
    float4 e = ez_c;
    const bool f9 = !GEN || (x >= n + 1 && x < nx - n && y >= n + 1 && y < ny - n);
    const float4 dhy = hyn - hyl;
    const float4 dhx = hxn - hx_prev;
    if (f9) {
      const float2 c = __ldg(reinterpret_cast<const float2*>(p.coef) + cell);
      float4 curl = dhy * f4(p.inv_dx) - dhx * f4(p.inv_dx);
      float4 en = c.x * e + c.y * curl;
      if constexpr (ND + NL > 0) en = ade_update<ND, NL>(p, cell, l, en, e, c.y);
      e = en;
    }
    if (GEN && n > 0) {
      // E-CPML x strips (fdtd_2d_batched.py:355-378)
      int sx = -1, ci = 0;
      if (y >= 1) {
        if (x >= 1 && x <= n) { sx = x - 1; ci = x - 1; }
        else if (x >= nx - n) { sx = n + (x - (nx - n)); ci = nx - 1 - x; }
      }
      if (sx >= 0) {
        float4* pp = p.psi_ezx + ((size_t)y * (2 * n) + sx) * p.lanes + l;
        float4 psi = p.cpml_b[ci] * (*pp) + p.cpml_c[ci] * (dhy * f4(p.inv_dx));
        *pp = psi;
        e = fma4(__ldg(p.dteps + cell), psi, e);
      }
      // E-CPML y strips (fdtd_2d_batched.py:380-406)
      int sy = -1;
      if (x >= 1) {
        if (y >= 1 && y <= n) { sy = y - 1; ci = y - 1; }
        else if (y >= ny - n) { sy = n + (y - (ny - n)); ci = ny - 1 - y; }
      }
      if (sy >= 0) {
        float4* pp = p.psi_ezy + ((size_t)sy * nx + x) * p.lanes + l;
        float4 psi = p.cpml_b[ci] * (*pp) + p.cpml_c[ci] * (dhx * f4(p.inv_dx));
        *pp = psi;
        e = fma4(-__ldg(p.dteps + cell), psi, e);
      }
    }
    if (GEN && (x == 0 || x == nx - 1 || y == 0 || y == ny - 1)) e = f4(0.f);

    // soft source and probe record (fdtd_2d_batched.py:509-526)
    const uint8_t flags = __ldg(p.row_flags + y);
    if (flags) {
      if (flags & 1) {
        const float w = __ldg(p.waveform + step);
        for (int s = 0; s < p.ntx; ++s) {
          if ((s >> 2) == l && __ldg(p.src_xy + 2 * s) == x && __ldg(p.src_xy + 2 * s + 1) == y)
            add_comp(e, s & 3, w);
        }
      }
      if (flags & 2) {
        for (int q = 0; q < p.nprobe; ++q) {
          if (__ldg(p.prb_xy + 2 * q) == x && __ldg(p.prb_xy + 2 * q + 1) == y) {
#pragma unroll
            for (int c = 0; c < 4; ++c) {
              const int tx = 4 * l + c;
              if (tx < p.ntx) p.probes[((size_t)tx * p.nprobe + q) * p.nsteps + step] = comp(e, c);
            }
          }
        }
      }
    }
    st4(ezw + at, e);

    hx_prev = hxn;
    ez_c = ez_up;
  }
}

template <int L, int ND, int NL>
__global__ void __launch_bounds__(kThreads2d) fdtd2d_step_kernel(const Fdtd2dParams p, int step, int par) {
  constexpr int CX = kThreads2d / L;  // cells per block along x
  const int x0 = blockIdx.x * CX;
  const int x = x0 + threadIdx.x / L;
  const int l = blockIdx.z * L + threadIdx.x % L;
  const int y0 = blockIdx.y * p.rows;
  const int y1 = min(y0 + p.rows, p.ny);
  if (x >= p.nx) return;
  const int n = p.n;
  // Block-uniform: every cell (and every recomputed halo H) of this block lies
  // in the plain interior of all regions.
  // (the far column/row is excluded too: Hy(nx-1), Hx(ny-1) are never updated
  // and Ez there is an edge).
  const int m = n > 1 ? n : 1;
  const bool interior = (x0 >= n + 1) && (x0 + CX <= p.nx - m) && (y0 >= n + 1) && (y1 <= p.ny - m);
  if (interior)
    column_segment<L, false, ND, NL>(p, x, l, y0, y1, step, par);
  else
    column_segment<L, true, ND, NL>(p, x, l, y0, y1, step, par);
}

// ------------------------------------------------------------------------
template <int L, int ND, int NL>
static cudaError_t launch_l(const Fdtd2dParams& p, int step, int par, cudaStream_t s) {
  constexpr int CX = kThreads2d / L;
  dim3 grid((p.nx + CX - 1) / CX, (p.ny + p.rows - 1) / p.rows, p.lanes / L);
  fdtd2d_step_kernel<L, ND, NL><<<grid, kThreads2d, 0, s>>>(p, step, par);
  return cudaGetLastError();
}

template <int ND, int NL>
static cudaError_t launch_ade(const Fdtd2dParams& p, int step, int par, cudaStream_t s) {
  switch (p.lanes_per_group) {
    case 1: return launch_l<1, ND, NL>(p, step, par, s);
    case 2: return launch_l<2, ND, NL>(p, step, par, s);
    case 4: return launch_l<4, ND, NL>(p, step, par, s);
    default: return launch_l<8, ND, NL>(p, step, par, s);
  }
}

cudaError_t fdtd2d_launch_step(const Fdtd2dParams& p, int step, int par, cudaStream_t s) {
  const int key = p.n_debye * 3 + p.n_lorentz;
  switch (key) {
    case 0: return launch_ade<0, 0>(p, step, par, s);
    case 1: return launch_ade<0, 1>(p, step, par, s);
    case 2: return launch_ade<0, 2>(p, step, par, s);
    case 3: return launch_ade<1, 0>(p, step, par, s);
    case 4: return launch_ade<1, 1>(p, step, par, s);
    case 6: return launch_ade<2, 0>(p, step, par, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ceep

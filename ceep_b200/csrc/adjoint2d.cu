// Exact discrete adjoint of the fused 2D step (sm_100a).
//
// The forward step (fdtd2d.cu, after fdtd_2d_batched.py:454-526) is a chain
// of linear maps; its transpose, applied in reverse order, is split into two
// launches per step:
//
//   A  E-phase adjoint (pointwise): probe gradient injection, edge zeroing,
//      transposed E-CPML psi recurrences, transposed interior E update and
//      Debye current recurrence.  Writes the adjoints of the two curls (cy of
//      Hy(x)-Hy(x-1), cx of Hx(y)-Hx(y-1)) and the pointwise part of the E
//      adjoint to scratch, and adds this step's per-cell parameter gradients:
//        dE1/dca = E^n, dE1/dcb = (E1 - ca E^n)/cb, dJ'/dk1 = J^n,
//        dJ'/dk2 = (E1 - E^n)/dt, dE1/dgamma = -cb J^n,
//      where E1 is the interior update (E^{n+1} minus the source).
//   B  H-phase adjoint (5-point gather): transposed curls, transposed H
//      updates including the strip psi recurrences, and the gather of the
//      E adjoint from the H differences E(x+1)-E(x), E(y+1)-E(y).
//
// Gradients are exact for the interior E region (where the update
// coefficients act); the E-CPML scale dt/(eps_r eps0) of strip cells is not
// differentiated (the ADE and phantom live in the interior by construction).
#include "../../include/ceep_b200.h"
#include "adjoint2d.cuh"
#include "common.cuh"

namespace ceep {

constexpr int kAdjThreads = 256;

template <int L>
CEEP_D float lane_sum(float v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
CEEP_D float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

// ---------------------------------------------------------------------------
template <int L, int ND>
__global__ void __launch_bounds__(kAdjThreads) adjoint2d_e_kernel(const Adjoint2dParams a, int step,
                                                                  const float4* __restrict__ ez_n,
                                                                  const float4* __restrict__ ez_np1,
                                                                  const float4* __restrict__ j_n) {
  const Fdtd2dParams& p = a.f;
  const int nx = p.nx, ny = p.ny, n = p.n;
  const long long total = (long long)p.groups * ny * nx * L;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  // Threads past the end still take part in the lane reductions (whole warps).
  const bool valid = id < total;
  const long long idc = valid ? id : total - 1;
  const int lo = (int)(idc % L);
  const long long cell_g = idc / L;
  const int x = (int)(cell_g % nx);
  const int y = (int)((cell_g / nx) % ny);
  const int g = (int)(cell_g / ((long long)nx * ny));
  const size_t cell = (size_t)y * nx + x;
  const size_t plane = (size_t)nx * ny;
  const int lane_g = g * L + lo;
  const float4 cf = __ldg(reinterpret_cast<const float4*>(p.coef) + cell);  // ca, cb, dt/eps
  const float inv = p.inv_dx;

  float4 E = a.ez[idc];
  // probe gradient injection: p_n = E after step n at the probe cells
  if (__ldg(p.row_flags + y) & 2) {
    for (int q = 0; q < p.nprobe; ++q)
      if (__ldg(p.prb_xy + 2 * q) == x && __ldg(p.prb_xy + 2 * q + 1) == y) {
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const int tx = 4 * lane_g + c;
          if (tx < p.ntx) add_comp(E, c, __ldg(a.probe_grad + ((size_t)tx * p.nprobe + q) * p.nsteps + step));
        }
      }
  }
  if (x == 0 || x == nx - 1 || y == 0 || y == ny - 1) E = f4(0.f);

  float4 cyv = f4(0.f), cxv = f4(0.f), elin = E;
  const size_t gy = (size_t)g * p.gs_psi_y, gx = (size_t)g * p.gs_psi_x;
  if (n > 0) {
    // transposed E-CPML, y strips: PEY' = b PEY + c inv cX ; E3 = E2 - dteps PEY'
    int sy = -1, ci = 0;
    if (x >= 1) {
      if (y >= 1 && y <= n) { sy = y - 1; ci = y - 1; }
      else if (y >= ny - n) { sy = n + (y - (ny - n)); ci = ny - 1 - y; }
    }
    if (sy >= 0) {
      float4* pp = a.psi_ezy + gy + ((size_t)sy * nx + x) * L + lo;
      const float4 tot = *pp - cf.z * E;
      if (valid) *pp = p.cpml_b[ci] * tot;
      cxv = (p.cpml_c[ci] * inv) * tot;
    }
    // transposed E-CPML, x strips: PEX' = b PEX + c inv cY ; E2 = E1 + dteps PEX'
    int sx = -1;
    if (y >= 1) {
      if (x >= 1 && x <= n) { sx = x - 1; ci = x - 1; }
      else if (x >= nx - n) { sx = n + (x - (nx - n)); ci = nx - 1 - x; }
    }
    if (sx >= 0) {
      float4* pp = a.psi_ezx + gx + ((size_t)y * 2 * n + sx) * L + lo;
      const float4 tot = *pp + cf.z * E;
      if (valid) *pp = p.cpml_b[ci] * tot;
      cyv = (p.cpml_c[ci] * inv) * tot;
    }
  }
  const bool f9 = x >= n + 1 && x < nx - n && y >= n + 1 && y < ny - n;
  const bool atomic = p.groups > 1;
  const size_t gstride = plane;
  float gv[2 + 3 * ND];
#pragma unroll
  for (int k = 0; k < 2 + 3 * ND; ++k) gv[k] = 0.f;
  if (f9) {
    // E1 = ca E + cb inv (cY - cX) - cb sum(gamma J);  J' = k1 J + k2 (E1 - E)/dt
    float4 e1 = ez_np1[idc];
    if (__ldg(p.row_flags + y) & 1) {  // the forward added the source after E1
      const float w = __ldg(p.waveform + step);
      for (int s = 0; s < p.ntx; ++s)
        if ((s >> 2) == lane_g && __ldg(p.src_xy + 2 * s) == x && __ldg(p.src_xy + 2 * s + 1) == y)
          add_comp(e1, s & 3, -w);
    }
    const float4 en = ez_n[idc];
    float4 e1tot = E;
    float4 jin[ND > 0 ? ND : 1], jn[ND > 0 ? ND : 1];
    float4 kq[ND > 0 ? ND : 1];
#pragma unroll
    for (int q = 0; q < ND; ++q) {
      kq[q] = __ldg(reinterpret_cast<const float4*>(p.ade_coef) + q * plane + cell);
      const size_t ja = (size_t)g * p.gs_j + (q * plane + cell) * L + lo;
      jin[q] = a.j[ja];
      jn[q] = j_n[ja];
      e1tot = fma4(kq[q].y * p.inv_dt, jin[q], e1tot);
    }
    elin = cf.x * e1tot;
#pragma unroll
    for (int q = 0; q < ND; ++q) {
      elin = fma4(-kq[q].y * p.inv_dt, jin[q], elin);
      const size_t ja = (size_t)g * p.gs_j + (q * plane + cell) * L + lo;
      if (valid) a.j[ja] = kq[q].x * jin[q] - (cf.y * kq[q].z) * e1tot;
    }
    cyv = (cf.y * inv) * e1tot;
    cxv = (-cf.y * inv) * e1tot;
    // parameter gradients of this step (this thread's four transmit events)
    gv[0] = dot4(e1tot, en);
    gv[1] = dot4(e1tot, (e1 - cf.x * en)) / cf.y;
#pragma unroll
    for (int q = 0; q < ND; ++q) {
      gv[2 + 3 * q] = dot4(jin[q], jn[q]);
      gv[3 + 3 * q] = dot4(jin[q], (e1 - en) * f4(p.inv_dt));
      gv[4 + 3 * q] = -cf.y * dot4(e1tot, jn[q]);
    }
  }
  // Sum over the L threads of the cell (warp-uniform: every lane of the warp
  // runs the shuffles); the first thread of the cell adds to the accumulator.
#pragma unroll
  for (int k = 0; k < 2 + 3 * ND; ++k) {
    const float v = lane_sum<L>(valid ? gv[k] : 0.f);
    if (valid && f9 && lo == 0) {
      double* dst = a.g + (size_t)k * gstride + cell;
      if (atomic)
        atomicAdd(dst, (double)v);
      else
        *dst += (double)v;
    }
  }
  if (valid) {
    a.cy[idc] = cyv;
    a.cx[idc] = cxv;
    a.elin[idc] = elin;
  }
}

// ---------------------------------------------------------------------------
// H-phase adjoint.  u_y(c) = A_y Y'* + kappa_x PHY'*, u_x(c) = -A_x X'* + kappa_y PHX'*
// are the adjoints of E(c+x)-E(c) and E(c+y)-E(c).
// ---------------------------------------------------------------------------
struct HAdjoint {
  float4 tot;   // adjoint of H' (total)
  float4 psi;   // adjoint of the old psi (written back)
  float4 u;     // adjoint of the forward difference
  bool strip;
};

CEEP_D HAdjoint hy_adjoint(const Fdtd2dParams& p, int x, int y, float4 yin, float4 cy_c, float4 cy_r,
                           float4 psi_in) {
  HAdjoint r;
  r.tot = yin + cy_c - cy_r;
  const int n = p.n;
  const float A = (x >= n && x < p.nx - 1 && y >= n && y < p.ny - n) ? p.db_dx : 0.f;
  int ci = -1;
  if (x < n) ci = x;
  else if (x >= p.nx - n && x < p.nx - 1) ci = p.nx - 1 - x;
  r.strip = ci >= 0;
  r.u = A * r.tot;
  r.psi = psi_in;
  if (r.strip) {
    const float4 pt = fma4(p.db, r.tot, psi_in);
    r.psi = p.cpml_b[ci] * pt;
    r.u = fma4(p.cpml_c[ci] * p.inv_dx, pt, r.u);
  }
  return r;
}

CEEP_D HAdjoint hx_adjoint(const Fdtd2dParams& p, int x, int y, float4 xin, float4 cx_c, float4 cx_u,
                           float4 psi_in) {
  HAdjoint r;
  r.tot = xin + cx_c - cx_u;
  const int n = p.n;
  const float A = (x >= n && x < p.nx - n && y >= n && y < p.ny - 1) ? p.db_dx : 0.f;
  int ci = -1;
  if (y < n) ci = y;
  else if (y >= p.ny - n && y < p.ny - 1) ci = p.ny - 1 - y;
  r.strip = ci >= 0;
  r.u = -A * r.tot;
  r.psi = psi_in;
  if (r.strip) {
    const float4 pt = fma4(-p.db, r.tot, psi_in);
    r.psi = p.cpml_b[ci] * pt;
    r.u = fma4(p.cpml_c[ci] * p.inv_dx, pt, r.u);
  }
  return r;
}

template <int L>
__global__ void __launch_bounds__(kAdjThreads) adjoint2d_h_kernel(const Adjoint2dParams a, int par) {
  const Fdtd2dParams& p = a.f;
  const int nx = p.nx, ny = p.ny, n = p.n;
  const long long total = (long long)p.groups * ny * nx * L;
  const long long id = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (id >= total) return;
  const int lo = (int)(id % L);
  const long long cell_g = id / L;
  const int x = (int)(cell_g % nx);
  const int y = (int)((cell_g / nx) % ny);
  const int g = (int)(cell_g / ((long long)nx * ny));
  const size_t sxs = L, sys = (size_t)nx * L;
  const size_t gx = (size_t)g * p.gs_psi_x, gy = (size_t)g * p.gs_psi_y;
  const float4* yin = a.hy[par];
  const float4* xin = a.hx[par];
  const float4 zero = f4(0.f);
  auto psi_y_at = [&](int xx, int yy) -> size_t {  // x-strip psi slot of cell (xx, yy), or ~0
    if (n == 0) return ~(size_t)0;
    if (xx < n) return gx + ((size_t)yy * 2 * n + xx) * L + lo;
    if (xx >= nx - n && xx < nx - 1) return gx + ((size_t)yy * 2 * n + n + (xx - (nx - n))) * L + lo;
    return ~(size_t)0;
  };
  auto psi_x_at = [&](int xx, int yy) -> size_t {  // y-strip psi slot, or ~0
    if (n == 0) return ~(size_t)0;
    if (yy < n) return gy + ((size_t)yy * nx + xx) * L + lo;
    if (yy >= ny - n && yy < ny - 1) return gy + ((size_t)(n + (yy - (ny - n))) * nx + xx) * L + lo;
    return ~(size_t)0;
  };

  const float4 cy_c = a.cy[id];
  const float4 cx_c = a.cx[id];
  // this cell
  const size_t py = psi_y_at(x, y), px = psi_x_at(x, y);
  const HAdjoint ry = hy_adjoint(p, x, y, yin[id], cy_c, x + 1 < nx ? a.cy[id + sxs] : zero,
                                 py != ~(size_t)0 ? a.psi_hy[par][py] : zero);
  const HAdjoint rx = hx_adjoint(p, x, y, xin[id], cx_c, y + 1 < ny ? a.cx[id + sys] : zero,
                                 px != ~(size_t)0 ? a.psi_hx[par][px] : zero);
  a.hy[par ^ 1][id] = ry.tot;
  a.hx[par ^ 1][id] = rx.tot;
  if (ry.strip) a.psi_hy[par ^ 1][py] = ry.psi;
  if (rx.strip) a.psi_hx[par ^ 1][px] = rx.psi;
  // neighbours' forward differences that involve this cell's E
  float4 e = a.elin[id] - ry.u - rx.u;
  if (x >= 1) {
    const size_t pyl = psi_y_at(x - 1, y);
    const HAdjoint l = hy_adjoint(p, x - 1, y, yin[id - sxs], a.cy[id - sxs], cy_c,
                                  pyl != ~(size_t)0 ? a.psi_hy[par][pyl] : zero);
    e = e + l.u;
  }
  if (y >= 1) {
    const size_t pxd = psi_x_at(x, y - 1);
    const HAdjoint d = hx_adjoint(p, x, y - 1, xin[id - sys], a.cx[id - sys], cx_c,
                                  pxd != ~(size_t)0 ? a.psi_hx[par][pxd] : zero);
    e = e + d.u;
  }
  a.ez[id] = e;
}

// ---------------------------------------------------------------------------
template <int L, int ND>
static cudaError_t launch_l(const Adjoint2dParams& a, int step, int par, const float4* ez_n, const float4* ez_np1,
                            const float4* j_n, cudaStream_t s) {
  const long long total = (long long)a.f.groups * a.f.ny * a.f.nx * L;
  const unsigned blocks = (unsigned)((total + kAdjThreads - 1) / kAdjThreads);
  adjoint2d_e_kernel<L, ND><<<blocks, kAdjThreads, 0, s>>>(a, step, ez_n, ez_np1, j_n);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  adjoint2d_h_kernel<L><<<blocks, kAdjThreads, 0, s>>>(a, par);
  return cudaGetLastError();
}

template <int ND>
static cudaError_t launch_nd(const Adjoint2dParams& a, int step, int par, const float4* ez_n, const float4* ez_np1,
                             const float4* j_n, cudaStream_t s) {
  switch (a.f.L) {
    case 1: return launch_l<1, ND>(a, step, par, ez_n, ez_np1, j_n, s);
    case 2: return launch_l<2, ND>(a, step, par, ez_n, ez_np1, j_n, s);
    case 4: return launch_l<4, ND>(a, step, par, ez_n, ez_np1, j_n, s);
    default: return launch_l<8, ND>(a, step, par, ez_n, ez_np1, j_n, s);
  }
}

cudaError_t adjoint2d_launch_step(const Adjoint2dParams& a, int step, int par, const float4* ez_n,
                                  const float4* ez_np1, const float4* j_n, cudaStream_t s) {
  if (a.f.n_lorentz != 0) return cudaErrorInvalidValue;
  switch (a.f.n_debye) {
    case 0: return launch_nd<0>(a, step, par, ez_n, ez_np1, j_n, s);
    case 1: return launch_nd<1>(a, step, par, ez_n, ez_np1, j_n, s);
    case 2: return launch_nd<2>(a, step, par, ez_n, ez_np1, j_n, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ceep

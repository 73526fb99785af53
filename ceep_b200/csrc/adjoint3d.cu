// Exact discrete adjoint of the batched 3D step (sm_100a): three launches per
// step, mirroring the forward's H and E half-steps.
//
// What the probe series depends on.  The forward (fdtd3d.cu, after
// fdtd_3d_batched.py:886-985) updates E only on the interior box
// [n+1, N-n)^3.  There it reads H on [n, N-n)^3, and no cell of that box lies
// on a CPML face (faces are x < n or x >= nx-n, likewise in y and z), so those
// H cells only ever take the plain box update, which reads E on [n, N-n]^3:
// interior E, or E cells the step never changes.  As a function of the
// material coefficients the probe series is therefore the Yee scheme on the
// interior with the surrounding E held fixed, and its exact transpose involves
// neither the CPML psi nor any H outside [n, N-n)^3.  This needs n >= 1.
//
// Forward step on those cells (D: the forward-difference curl of the H
// update, C: the backward-difference curl of the E update):
//   H'   = da H + db D(E)
//   E'   = ca E + cb (C(H') - sum_q gamma_q J_q)        (+ w at source cells)
//   J_q' = k1_q J_q + k2_q (E' - E) / dt
// Transposed, with mu = adj(E') + sum_q (k2_q/dt) adj(J_q') (state `mu`) and
// nu such that adj(H') = da nu_next (state `nu`, the da factor applied when
// it is read):
//   kernel 1 on [n, N-n)^3:     nu = da nu_next - D(cb mu)
//   kernel 2 on [n+1, N-n)^3:   adj(E)   = ca mu - sum_q (k2_q/dt) adj(J_q') - C(db nu)
//                               adj(J_q) = k1_q adj(J_q') - gamma_q cb mu
//                               mu_prev  = adj(E) + sum_q (k2_q/dt) adj(J_q)
// mu is zero outside the interior (nothing writes it there), so kernel 1
// needs no region tests.  Kernel 2 also adds this step's per-cell gradients,
// summed over the three components and the TX of the cell's group:
//   d/dca += mu . E^n,   d/dcb += mu . (E1 - ca E^n) / cb,
//   d/dk2_q += adj(J_q') . (E1 - E^n) / dt,
// E1 being the update before the source.  A one-block kernel ahead of
// kernel 1 adds dLoss/dprobe to mu_z at the (interior) probe cells.
#include "../../include/ceep_b200.h"
#include "adjoint3d.cuh"
#include "common.cuh"

namespace ceep {

constexpr int kAdj3dThreads = 128;

template <int L>
CEEP_D float lane_sum3(float v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
CEEP_D float dot4_3(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }

// dLoss/dprobe of this step into mu_z; one thread per TX walks the probes in
// order, so repeated probe cells add in a fixed order.
__global__ void adjoint3d_inject_kernel(const Adjoint3dParams a, int step) {
  const Fdtd3dParams& p = a.f;
  const int n = p.n;
  float* mz = reinterpret_cast<float*>(a.mu + 2 * a.cs);
  for (int b = threadIdx.x; b < p.ntx; b += blockDim.x) {
    const int g = b / (4 * p.L), lane = b % (4 * p.L);
    for (int q = 0; q < p.nprobe; ++q) {
      const int x = p.prb_xyz[3 * q], y = p.prb_xyz[3 * q + 1], z = p.prb_xyz[3 * q + 2];
      if (x < n + 1 || x >= p.nx - n || y < n + 1 || y >= p.ny - n || z < n + 1 || z >= p.nz - n) continue;
      const size_t cell = ((size_t)z * p.ny + y) * p.nx + x;
      mz[4 * ((size_t)g * p.gs_field + cell * p.L) + lane] +=
          a.probe_grad[((size_t)b * p.nprobe + q) * p.nsteps + step];
    }
  }
}

// Kernel 1: nu = da nu_next - D(cb mu) on [n, N-n)^3.  A block is one x-row
// of 128/L cells; each thread walks a z segment carrying cb mu of the plane
// above into the next iteration.
template <int L>
__global__ void __launch_bounds__(kAdj3dThreads, 6) adjoint3d_h_kernel(const Adjoint3dParams a) {
  constexpr int CX = kAdj3dThreads / L;
  const Fdtd3dParams& p = a.f;
  const int n = p.n, nx = p.nx, ny = p.ny, nz = p.nz;
  const int x = n + blockIdx.x * CX + threadIdx.x / L;
  const int lo = threadIdx.x % L;
  const int y = n + blockIdx.y;
  const int zseg = blockIdx.z % a.zsegs_h, g = blockIdx.z / a.zsegs_h;
  const int z0 = n + zseg * p.zrows, z1 = min(z0 + p.zrows, nz - n);
  if (x >= nx - n) return;
  const size_t sx = L, sy = (size_t)nx * L, sz = (size_t)ny * nx * L, cs = a.cs;
  const size_t cz = (size_t)ny * nx;
  const float4* __restrict__ mu = a.mu + (size_t)g * p.gs_field;
  float4* nu = a.nu + (size_t)g * p.gs_field;
  const float4* coef = reinterpret_cast<const float4*>(p.coef);  // da, db, ca, cb
  const float4 inv = f4(p.inv_dx);
  size_t at = (size_t)z0 * sz + (size_t)y * sy + (size_t)x * sx + lo;
  size_t cc = (size_t)z0 * cz + (size_t)y * nx + x;
  const float cb = __ldg(coef + cc).w;
  float4 mx = cb * ld4(mu + at), my = cb * ld4(mu + cs + at), mz = cb * ld4(mu + 2 * cs + at);
  for (int z = z0; z < z1; ++z, at += sz, cc += cz) {
    const float da = __ldg(coef + cc).x;
    // the +z, +y and +x neighbours lie in [n, N-n], inside the grid since n >= 1
    const float cbz = __ldg(coef + cc + cz).w;
    const float4 mxz = cbz * ld4(mu + at + sz), myz = cbz * ld4(mu + cs + at + sz);
    const float4 mzz = cbz * ld4(mu + 2 * cs + at + sz);
    const float cby = __ldg(coef + cc + nx).w;
    const float4 mxy = cby * ld4(mu + at + sy), mzy = cby * ld4(mu + 2 * cs + at + sy);
    const float cbx = __ldg(coef + cc + 1).w;
    const float4 myx = cbx * ld4(mu + cs + at + sx), mzx = cbx * ld4(mu + 2 * cs + at + sx);
    float4* vx = nu + at;
    float4* vy = nu + cs + at;
    float4* vz = nu + 2 * cs + at;
    *vx = da * *vx - ((myz - my) * inv - (mzy - mz) * inv);
    *vy = da * *vy - ((mzx - mz) * inv - (mxz - mx) * inv);
    *vz = da * *vz - ((mxy - mx) * inv - (myx - my) * inv);
    mx = mxz;
    my = myz;
    mz = mzz;
  }
}

// Kernel 2: the transposed E update and current recurrences on the interior,
// with the per-cell gradients.  Threads past the row end load a valid cell
// (the last interior column) so that every lane joins the lane sums; they
// store nothing.
template <int L, int ND>
__global__ void __launch_bounds__(kAdj3dThreads, 4)
    adjoint3d_e_kernel(const Adjoint3dParams a, int step, const float4* __restrict__ e_n,
                       const float4* __restrict__ e_np1, int e_n_post) {
  constexpr int CX = kAdj3dThreads / L;
  constexpr int KS = 2 + ND;
  const Fdtd3dParams& p = a.f;
  const int n = p.n, nx = p.nx, ny = p.ny, nz = p.nz;
  const int xr = n + 1 + blockIdx.x * CX + threadIdx.x / L;
  const int lo = threadIdx.x % L;
  const int y = n + 1 + blockIdx.y;
  const int zseg = blockIdx.z % a.zsegs_e, g = blockIdx.z / a.zsegs_e;
  const int z0 = n + 1 + zseg * p.zrows, z1 = min(z0 + p.zrows, nz - n);
  const bool live = xr < nx - n;
  const int x = live ? xr : nx - n - 1;
  const size_t sx = L, sy = (size_t)nx * L, sz = (size_t)ny * nx * L, cs = a.cs;
  const size_t cz = (size_t)ny * nx, cells = (size_t)nz * ny * nx;
  const size_t goff = (size_t)g * p.gs_field;
  float4* mu = a.mu + goff;
  const float4* __restrict__ nu = a.nu + goff;
  // the saved slots cover the interior box only: (3, G, nzi, nyi, nxi, L)
  const size_t scs = (size_t)p.save_cs;
  float4* lj = a.lj + (size_t)g * p.gs_j;
  const float4* coef = reinterpret_cast<const float4*>(p.coef);
  const float4* ade = reinterpret_cast<const float4*>(p.ade_coef);
  const float4 inv = f4(p.inv_dx);
  const float inv_dt = p.inv_dt;
  // the saved E^n lacks the source of the previous step at this thread's
  // own source cells (its four TX at (x, y)); the forward added it with one
  // FP32 add, repeated here
  int zsrc[4] = {-1, -1, -1, -1};
  float wprev = 0.f;
  if (!e_n_post && step > 0) {
    wprev = __ldg(p.waveform + step - 1);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const int b = g * 4 * L + 4 * lo + k;
      if (b < p.ntx && __ldg(p.src_xyz + 3 * b) == x && __ldg(p.src_xyz + 3 * b + 1) == y)
        zsrc[k] = __ldg(p.src_xyz + 3 * b + 2);
    }
  }
  const int nxi = nx - 2 * n - 1, nyi = ny - 2 * n - 1;
  double* gw = a.g + (size_t)g * KS * a.icells + ((size_t)(z0 - n - 1) * nyi + (y - n - 1)) * nxi + (x - n - 1);
  const size_t s_at0 = (size_t)g * a.icells * L + (((size_t)(z0 - n - 1) * nyi + (y - n - 1)) * nxi + (x - n - 1)) * L + lo;
  const float4* __restrict__ en = e_n + s_at0;
  const float4* __restrict__ e1 = e_np1 + s_at0;
  const size_t s_sz = (size_t)nyi * nxi * L;
  size_t at = (size_t)z0 * sz + (size_t)y * sy + (size_t)x * sx + lo;
  size_t cc = (size_t)z0 * cz + (size_t)y * nx + x;
  // db nu of the plane below (x and y components)
  const float dbm = __ldg(coef + cc - cz).y;
  float4 nxm = dbm * ld4(nu + at - sz), nym = dbm * ld4(nu + cs + at - sz);
  for (int z = z0; z < z1; ++z, at += sz, cc += cz, gw += (size_t)nyi * nxi, en += s_sz, e1 += s_sz) {
    const float4 cf = __ldg(coef + cc);
    const float4 Nx = cf.y * ld4(nu + at), Ny = cf.y * ld4(nu + cs + at), Nz = cf.y * ld4(nu + 2 * cs + at);
    const float dby = __ldg(coef + cc - nx).y;
    const float4 Nxy = dby * ld4(nu + at - sy), Nzy = dby * ld4(nu + 2 * cs + at - sy);
    const float dbx = __ldg(coef + cc - 1).y;
    const float4 Nyx = dbx * ld4(nu + cs + at - sx), Nzx = dbx * ld4(nu + 2 * cs + at - sx);
    const float4 curl[3] = {(Nz - Nzy) * inv - (Ny - nym) * inv, (Nx - nxm) * inv - (Nz - Nzx) * inv,
                            (Ny - Nyx) * inv - (Nx - Nxy) * inv};
    float4 kq[ND > 0 ? ND : 1];
#pragma unroll
    for (int q = 0; q < ND; ++q) kq[q] = __ldg(ade + q * cells + cc);  // k1, k2, gamma, 0
    float gv[KS];
#pragma unroll
    for (int k = 0; k < KS; ++k) gv[k] = 0.f;
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const size_t ac = c * cs + at;
      const float4 m = mu[ac];
      float4 E0 = ld4(en + c * scs);
      const float4 E1 = ld4(e1 + c * scs);
      if (c == 2) {
#pragma unroll
        for (int k = 0; k < 4; ++k)
          if (zsrc[k] == z) add_comp(E0, k, wprev);
      }
      float4 le = cf.z * m - curl[c];
      gv[0] += dot4_3(m, E0);
      gv[1] += dot4_3(m, E1 - cf.z * E0);
      float4 mnew = f4(0.f);
#pragma unroll
      for (int q = 0; q < ND; ++q) {
        float4* jp = lj + ((size_t)(q * 3 + c) * cells + cc) * L + lo;
        const float4 lq = *jp;
        const float k2dt = kq[q].y * inv_dt;
        le = le - k2dt * lq;
        gv[2 + q] += dot4_3(lq, E1 - E0);
        const float4 lqn = kq[q].x * lq - (kq[q].z * cf.w) * m;
        mnew = mnew + k2dt * lqn;
        if (live) *jp = lqn;
      }
      if (live) mu[ac] = le + mnew;
    }
#pragma unroll
    for (int k = 0; k < KS; ++k) {
      float v = lane_sum3<L>(gv[k]);
      v = k == 1 ? v / cf.w : (k >= 2 ? v * inv_dt : v);
      if (live && (k % L) == lo) atomicAdd(gw + (size_t)k * a.icells, (double)v);
    }
    nxm = Nx;
    nym = Ny;
  }
}

template <int L, int ND>
static cudaError_t step_l(const Adjoint3dParams& a, int step, const float4* en, const float4* e1, bool post,
                          cudaStream_t s) {
  constexpr int CX = kAdj3dThreads / L;
  const Fdtd3dParams& p = a.f;
  if (p.nprobe) {
    adjoint3d_inject_kernel<<<1, 64, 0, s>>>(a, step);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  const int nh = p.nx - 2 * p.n, mh = p.ny - 2 * p.n;
  dim3 gh((nh + CX - 1) / CX, mh, a.zsegs_h * p.groups);
  adjoint3d_h_kernel<L><<<gh, kAdj3dThreads, 0, s>>>(a);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return e;
  const int ni = nh - 1, mi = mh - 1;
  dim3 ge((ni + CX - 1) / CX, mi, a.zsegs_e * p.groups);
  adjoint3d_e_kernel<L, ND><<<ge, kAdj3dThreads, 0, s>>>(a, step, en, e1, post ? 1 : 0);
  return cudaGetLastError();
}

template <int ND>
static cudaError_t step_nd(const Adjoint3dParams& a, int step, const float4* en, const float4* e1, bool post,
                           cudaStream_t s) {
  switch (a.f.L) {
    case 1: return step_l<1, ND>(a, step, en, e1, post, s);
    case 2: return step_l<2, ND>(a, step, en, e1, post, s);
    case 4: return step_l<4, ND>(a, step, en, e1, post, s);
    default: return step_l<8, ND>(a, step, en, e1, post, s);
  }
}

cudaError_t adjoint3d_launch_step(const Adjoint3dParams& a, int step, const float4* e_n, const float4* e_np1,
                                  bool e_n_post, cudaStream_t s) {
  switch (a.f.n_debye) {
    case 0: return step_nd<0>(a, step, e_n, e_np1, e_n_post, s);
    case 1: return step_nd<1>(a, step, e_n, e_np1, e_n_post, s);
    case 2: return step_nd<2>(a, step, e_n, e_np1, e_n_post, s);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ceep

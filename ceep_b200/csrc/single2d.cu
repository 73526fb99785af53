// Non-batched 2D FDTD (TMz / TEz) with CFS-CPML, PEC and Mur boundaries, for
// sm_100a: the reference's FDTD2D.step() (src/ceep/solvers/fdtd_base.py:158-190,
// src/ceep/solvers/fdtd_2d.py:111-260, src/ceep/boundaries/absorbing.py).
//
// One step is
//   H kernel   plain H update of every cell plus the CPML H corrections of
//              the strip cells (they read only E, so each cell finishes its
//              H values alone; absorbing.py:332-451)
//   E kernel   plain E update, the soft sources of E components at the cell
//              (list order), then the boundary operations in list order:
//              CPML E corrections (absorbing.py:453-561) and PEC zeroing
//              (absorbing.py:58-72).  E corrections read only H.
//   Hz-source  one thread adds TEz Hz sources in list order (Hz is read by
//              the neighbours' E updates, so it cannot be added inside the
//              E kernel)
//   Mur        one block: the first-order Mur update of the four edges of Ez
//              (TMz) or Hz (TEz) in the reference's order, x faces then y
//              faces (absorbing.py:126-166); last boundary operation only
//   record     probe / monitor cells into (nrec, nsteps), and a copy of the
//              snapshot field every snap_interval steps
// Fields are (nx, ny) FP32 with y fastest, the reference's layout.  All
// launches of a run are captured once into a CUDA graph and replayed.
#include <map>
#include <tuple>

#include "../../include/ceep_b200.h"
#include "capi_internal.h"
#include "common.cuh"

namespace ceep {

constexpr int kS2x = 32, kS2y = 8;  // threads per block along y (fastest) and x

struct Single2dParams {
  int nx, ny, mode, nsteps;
  float inv_dx, inv_dy, dt_mu0, dt_eps0, mur_kx, mur_ky;
  float* f[3];
  const float2* ce;  // ca, cb
  const float2* ch;  // da, db
  int n_ops, ops[4];
  int t;
  const float* cpml;  // be_x, ce_x, bh_x, ch_x, be_y, ce_y, bh_y, ch_y: t each
  float* psi;         // 4 x (t, ny): E x-lo, E x-hi, H x-lo, H x-hi; 4 x (nx, t): E/H y-lo/hi
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

template <int MODE, bool CPML>
__global__ void __launch_bounds__(kS2x * kS2y) single2d_h_kernel(const Single2dParams p) {
  const int j = blockIdx.x * kS2x + threadIdx.x;
  const int i = blockIdx.y * kS2y + threadIdx.y;
  const int nx = p.nx, ny = p.ny;
  if (i >= nx || j >= ny) return;
  const size_t c = (size_t)i * ny + j;
  const float2 d = __ldg(p.ch + c);
  const float* bhx = p.cpml + 2 * p.t;
  const float* chx = p.cpml + 3 * p.t;
  const float* bhy = p.cpml + 6 * p.t;
  const float* chy = p.cpml + 7 * p.t;
  float* psi_hx = p.psi + 2 * (size_t)p.t * ny;      // H x-lo, then H x-hi
  float* psi_hy = p.psi + 4 * (size_t)p.t * ny + 2 * (size_t)nx * p.t;  // H y-lo, then H y-hi
  if (MODE == 0) {
    // TMz: Hx (fdtd_2d.py:132-136), Hy (:139-142); CPML x strips act on Hy,
    // y strips on Hx (absorbing.py:413-451)
    const float* ez = p.f[0];
    float* hx = p.f[1];
    float* hy = p.f[2];
    const float e0 = __ldg(ez + c);
    const float dy = j + 1 < ny ? __ldg(ez + c + 1) - e0 : 0.f;
    const float dx = i + 1 < nx ? __ldg(ez + c + ny) - e0 : 0.f;
    float vx = hx[c], vy = hy[c];
    if (j < ny - 1) vx = d.x * vx - (d.y * p.inv_dy) * dy;
    if (i < nx - 1) vy = d.x * vy + (d.y * p.inv_dx) * dx;
    if (CPML) {
      const int t = p.t;
      const Strips sx = strips(i, nx, t, true);
      if (sx.lo >= 0) {
        float* q = psi_hx + (size_t)sx.lo * ny + j;
        const float v = bhx[sx.lo_k] * *q + chx[sx.lo_k] * dx * p.inv_dx;
        *q = v;
        vy += p.dt_mu0 * v;
      }
      if (sx.hi >= 0) {
        float* q = psi_hx + (size_t)(t + sx.hi) * ny + j;
        const float v = bhx[sx.hi] * *q + chx[sx.hi] * dx * p.inv_dx;
        *q = v;
        vy += p.dt_mu0 * v;
      }
      const Strips sy = strips(j, ny, t, true);
      if (sy.lo >= 0) {
        float* q = psi_hy + (size_t)i * t + sy.lo;
        const float v = bhy[sy.lo_k] * *q + chy[sy.lo_k] * dy * p.inv_dy;
        *q = v;
        vx -= p.dt_mu0 * v;
      }
      if (sy.hi >= 0) {
        float* q = psi_hy + (size_t)nx * t + (size_t)i * t + sy.hi;
        const float v = bhy[sy.hi] * *q + chy[sy.hi] * dy * p.inv_dy;
        *q = v;
        vx -= p.dt_mu0 * v;
      }
    }
    hx[c] = vx;
    hy[c] = vy;
  } else {
    // TEz: Hz (fdtd_2d.py:169-183); CPML x strips subtract, y strips add
    // (absorbing.py:355-405)
    float* hz = p.f[0];
    const float* ex = p.f[1];
    const float* ey = p.f[2];
    const float x0 = __ldg(ex + c), y0 = __ldg(ey + c);
    const float dex = j + 1 < ny ? __ldg(ex + c + 1) - x0 : 0.f;
    const float dey = i + 1 < nx ? __ldg(ey + c + ny) - y0 : 0.f;
    float v = hz[c];
    if (i < nx - 1 && j < ny - 1) v = d.x * v + d.y * (dex * p.inv_dy - dey * p.inv_dx);
    if (CPML) {
      const int t = p.t;
      const Strips sx = strips(i, nx, t, true);
      if (sx.lo >= 0) {
        float* q = psi_hx + (size_t)sx.lo * ny + j;
        const float w = bhx[sx.lo_k] * *q + chx[sx.lo_k] * dey * p.inv_dx;
        *q = w;
        v -= p.dt_mu0 * w;
      }
      if (sx.hi >= 0) {
        float* q = psi_hx + (size_t)(t + sx.hi) * ny + j;
        const float w = bhx[sx.hi] * *q + chx[sx.hi] * dey * p.inv_dx;
        *q = w;
        v -= p.dt_mu0 * w;
      }
      const Strips sy = strips(j, ny, t, true);
      if (sy.lo >= 0) {
        float* q = psi_hy + (size_t)i * t + sy.lo;
        const float w = bhy[sy.lo_k] * *q + chy[sy.lo_k] * dex * p.inv_dy;
        *q = w;
        v += p.dt_mu0 * w;
      }
      if (sy.hi >= 0) {
        float* q = psi_hy + (size_t)nx * t + (size_t)i * t + sy.hi;
        const float w = bhy[sy.hi] * *q + chy[sy.hi] * dex * p.inv_dy;
        *q = w;
        v += p.dt_mu0 * w;
      }
    }
    hz[c] = v;
  }
}

// CPML E correction of one strip side: psi' = b psi + c diff/d, returns psi'.
CEEP_D float psi_e(float* q, float b, float cc, float diff, float inv) {
  const float v = b * *q + cc * diff * inv;
  *q = v;
  return v;
}

template <int MODE, bool CPML>
__global__ void __launch_bounds__(kS2x * kS2y) single2d_e_kernel(const Single2dParams p, int step) {
  const int j = blockIdx.x * kS2x + threadIdx.x;
  const int i = blockIdx.y * kS2y + threadIdx.y;
  const int nx = p.nx, ny = p.ny;
  if (i >= nx || j >= ny) return;
  const size_t c = (size_t)i * ny + j;
  const float2 k = __ldg(p.ce + c);
  const int t = p.t;
  const float* bex = p.cpml;
  const float* cex = p.cpml + t;
  const float* bey = p.cpml + 4 * t;
  const float* cey = p.cpml + 5 * t;
  float* psi_ex = p.psi;                                  // E x-lo, then E x-hi: (t, ny)
  float* psi_ey = p.psi + 4 * (size_t)t * ny;             // E y-lo, then E y-hi: (nx, t)
  const bool edge = i == 0 || i == nx - 1 || j == 0 || j == ny - 1;
  if (MODE == 0) {
    // TMz: Ez on [1, nx) x [1, ny) (fdtd_2d.py:165-171)
    float* ez = p.f[0];
    const float* hx = p.f[1];
    const float* hy = p.f[2];
    const float hxc = __ldg(hx + c), hyc = __ldg(hy + c);
    const float dhy = i > 0 ? hyc - __ldg(hy + c - ny) : 0.f;
    const float dhx = j > 0 ? hxc - __ldg(hx + c - 1) : 0.f;
    float e = ez[c];
    if (i > 0 && j > 0) e = k.x * e + k.y * (dhy * p.inv_dx - dhx * p.inv_dy);
    for (int s = __ldg(p.src_row + i); s < __ldg(p.src_row + i + 1); ++s)  // fdtd_2d.py:245-260
      if (__ldg(p.src + 3 * s + 1) == j && __ldg(p.src + 3 * s + 2) == 0)
        e += __ldg(p.waveform + (size_t)s * p.nsteps + step);
    for (int o = 0; o < p.n_ops; ++o) {
      if (CPML && p.ops[o] == kOpCpml) {
        const Strips sx = strips(i, nx, t, false);
        if (sx.lo >= 0) e += p.dt_eps0 * psi_e(psi_ex + (size_t)sx.lo * ny + j, bex[sx.lo_k], cex[sx.lo_k], dhy, p.inv_dx);
        if (sx.hi >= 0) e += p.dt_eps0 * psi_e(psi_ex + (size_t)(t + sx.hi) * ny + j, bex[sx.hi], cex[sx.hi], dhy, p.inv_dx);
        const Strips sy = strips(j, ny, t, false);
        if (sy.lo >= 0) e -= p.dt_eps0 * psi_e(psi_ey + (size_t)i * t + sy.lo, bey[sy.lo_k], cey[sy.lo_k], dhx, p.inv_dy);
        if (sy.hi >= 0)
          e -= p.dt_eps0 * psi_e(psi_ey + (size_t)nx * t + (size_t)i * t + sy.hi, bey[sy.hi], cey[sy.hi], dhx, p.inv_dy);
      } else if (p.ops[o] == kOpPec && edge) {
        e = 0.f;
      }
    }
    ez[c] = e;
  } else {
    // TEz: Ex on j >= 1, Ey on i >= 1 (fdtd_2d.py:205-217)
    const float* hz = p.f[0];
    float* ex = p.f[1];
    float* ey = p.f[2];
    const float hc = __ldg(hz + c);
    const float dy = j > 0 ? hc - __ldg(hz + c - 1) : 0.f;
    const float dx = i > 0 ? hc - __ldg(hz + c - ny) : 0.f;
    float vx = ex[c], vy = ey[c];
    if (j > 0) vx = k.x * vx + (k.y * p.inv_dy) * dy;
    if (i > 0) vy = k.x * vy - (k.y * p.inv_dx) * dx;
    for (int s = __ldg(p.src_row + i); s < __ldg(p.src_row + i + 1); ++s) {
      if (__ldg(p.src + 3 * s + 1) != j) continue;
      const int fld = __ldg(p.src + 3 * s + 2);
      const float w = __ldg(p.waveform + (size_t)s * p.nsteps + step);
      if (fld == 1) vx += w;
      else if (fld == 2) vy += w;
    }
    for (int o = 0; o < p.n_ops; ++o) {
      if (CPML && p.ops[o] == kOpCpml) {
        // y strips on Ex first, then x strips on Ey (absorbing.py:467-511)
        const Strips sy = strips(j, ny, t, false);
        if (sy.lo >= 0) vx += p.dt_eps0 * psi_e(psi_ey + (size_t)i * t + sy.lo, bey[sy.lo_k], cey[sy.lo_k], dy, p.inv_dy);
        if (sy.hi >= 0)
          vx += p.dt_eps0 * psi_e(psi_ey + (size_t)nx * t + (size_t)i * t + sy.hi, bey[sy.hi], cey[sy.hi], dy, p.inv_dy);
        const Strips sx = strips(i, nx, t, false);
        if (sx.lo >= 0) vy -= p.dt_eps0 * psi_e(psi_ex + (size_t)sx.lo * ny + j, bex[sx.lo_k], cex[sx.lo_k], dx, p.inv_dx);
        if (sx.hi >= 0) vy -= p.dt_eps0 * psi_e(psi_ex + (size_t)(t + sx.hi) * ny + j, bex[sx.hi], cex[sx.hi], dx, p.inv_dx);
      } else if (p.ops[o] == kOpPec) {
        if (i == 0 || i == nx - 1) vx = 0.f;  // absorbing.py:68-72
        if (j == 0 || j == ny - 1) vy = 0.f;
      }
    }
    ex[c] = vx;
    ey[c] = vy;
  }
}

// TEz Hz sources, in list order (fdtd_2d.py:253-254).
__global__ void single2d_src_h_kernel(const Single2dParams p, int step) {
  if (threadIdx.x != 0) return;
  for (int s = 0; s < p.nsrc; ++s)
    if (p.src[3 * s + 2] == 0)
      p.f[0][(size_t)p.src[3 * s] * p.ny + p.src[3 * s + 1]] += p.waveform[(size_t)s * p.nsteps + step];
}

// First-order Mur on the edges of field 0 (absorbing.py:126-166).  prev holds
// the previous step's lines next to the edges (x0, xn: ny each; y0, yn: nx
// each); this step's lines go to the other half of the pair.
__global__ void single2d_mur_kernel(const Single2dParams p, int step) {
  const int nx = p.nx, ny = p.ny;
  float* e = p.f[0];
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

__global__ void single2d_record_kernel(const Single2dParams p, int step) {
  const int r = blockIdx.x * blockDim.x + threadIdx.x;
  if (r >= p.nrec) return;
  p.rec_out[(size_t)r * p.nsteps + step] = p.f[p.rec[2 * r + 1]][p.rec[2 * r]];
}

template <int MODE, bool CPML>
static cudaError_t step_t(const Single2dParams& p, int step, cudaStream_t s) {
  const dim3 blk(kS2x, kS2y), grd((p.ny + kS2x - 1) / kS2x, (p.nx + kS2y - 1) / kS2y);
  single2d_h_kernel<MODE, CPML><<<grd, blk, 0, s>>>(p);
  single2d_e_kernel<MODE, CPML><<<grd, blk, 0, s>>>(p, step);
  return cudaGetLastError();
}

}  // namespace ceep

struct ceep2s_plan {
  ceep::Single2dParams p;
  bool hz_src = false, mur = false, cpml = false;
  std::map<std::pair<int64_t, int64_t>, cudaGraphExec_t> graphs;
};

static int run_steps2s(const ceep2s_plan* pl, int64_t step0, int64_t nsteps, cudaStream_t s) {
  const ceep::Single2dParams& p = pl->p;
  for (int64_t k = 0; k < nsteps; ++k) {
    const int step = (int)(step0 + k);
    cudaError_t e;
    if (p.mode == 0)
      e = pl->cpml ? ceep::step_t<0, true>(p, step, s) : ceep::step_t<0, false>(p, step, s);
    else
      e = pl->cpml ? ceep::step_t<1, true>(p, step, s) : ceep::step_t<1, false>(p, step, s);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "single2d step launch");
    if (pl->hz_src) ceep::single2d_src_h_kernel<<<1, 32, 0, s>>>(p, step);
    if (pl->mur) ceep::single2d_mur_kernel<<<1, 1024, 0, s>>>(p, step);
    if (p.nrec) ceep::single2d_record_kernel<<<(p.nrec + 255) / 256, 256, 0, s>>>(p, step);
    e = cudaGetLastError();
    if (e != cudaSuccess) return ceep::cuda_fail(e, "single2d epilogue launch");
    if (p.snapshots && step % p.snap_interval == 0) {
      const size_t n = (size_t)p.nx * p.ny;
      e = cudaMemcpyAsync(p.snapshots + (size_t)(step / p.snap_interval) * n, p.f[p.snap_field], n * sizeof(float),
                          cudaMemcpyDeviceToDevice, s);
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
  if (!d->f0 || !d->f1 || !d->f2 || !d->coef_e || !d->coef_h)
    return fail(CEEP_ERR_INVALID, "null field or coefficient buffer");
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
  if (cpml && (d->cpml_t < 1 || !d->cpml || !d->psi)) return fail(CEEP_ERR_INVALID, "CPML: thickness/buffers");
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
  p.f[0] = d->f0; p.f[1] = d->f1; p.f[2] = d->f2;
  p.ce = reinterpret_cast<const float2*>(d->coef_e);
  p.ch = reinterpret_cast<const float2*>(d->coef_h);
  p.n_ops = d->n_ops;
  for (int o = 0; o < 4; ++o) p.ops[o] = o < d->n_ops ? d->ops[o] : 0;
  p.t = cpml ? d->cpml_t : 0;
  p.cpml = d->cpml; p.psi = d->psi; p.mur_prev = d->mur_prev;
  p.nsrc = d->nsrc; p.src = d->src; p.src_row = d->src_row; p.waveform = d->waveform;
  p.nrec = d->nrec; p.rec = d->rec; p.rec_out = d->rec_out;
  p.snap_field = d->snap_field; p.snap_interval = d->snap_interval > 0 ? d->snap_interval : 1;
  p.snapshots = d->snapshots;
  pl->cpml = cpml;
  pl->mur = mur;
  pl->hz_src = hz_src;
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
  if (!use_graph || s == nullptr) return run_steps2s(pl, step0, nsteps, s);
  auto key = std::make_pair(step0, nsteps);
  auto it = pl->graphs.find(key);
  if (it == pl->graphs.end()) {
    cudaGraph_t g;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "cudaStreamBeginCapture");
    int rc = run_steps2s(pl, step0, nsteps, s);
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
  return e == cudaSuccess ? CEEP_OK : ceep::cuda_fail(e, "cudaGraphLaunch");
}

extern "C" int ceep2s_plan_destroy(ceep2s_plan* pl) {
  if (!pl) return CEEP_OK;
  for (auto& kv : pl->graphs) cudaGraphExecDestroy(kv.second);
  delete pl;
  return CEEP_OK;
}

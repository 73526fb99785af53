// Batched 3D Yee FDTD for sm_100a: one H kernel and one E kernel per step
// (each a fused half-step), plus a one-block epilogue for sources/probes.
//
// Region semantics of the reference's BatchedFDTD3D.run()
// (src/ceep/solvers/fdtd_3d_batched.py:886-985):
//   H  interior boxes (:753-818):
//        Hx on x in [n, nx-n), y in [n, ny-1), z in [n, nz-1)
//        Hy on x in [n, nx-1), y in [n, ny-n), z in [n, nz-1)
//        Hz on x in [n, nx-1), y in [n, ny-1), z in [n, nz-n)
//      then the CPML faces in the order x, y, z (:398-586); each face's psi
//      recurrence runs over the whole slab, low faces use forward and high
//      faces backward differences:
//        x faces: Hy -= db psi(dEz/dx) (z < nz-1), Hz += db psi(dEy/dx) (y < ny-1)
//        y faces: Hx -= db psi(dEz/dy) (z < nz-1), Hz += db psi(dEx/dy) (x < nx-1)
//        z faces: Hx += db psi(dEy/dz) (y < ny-1), Hy -= db psi(dEx/dz) (x < nx-1)
//      each face update being H = da*H +/- db*psi on the already-updated H.
//   E  only on [n+1, N-n)^3 (:820-884); the rest of E is never updated.
//   E zeroed on the three low faces (:936-944), soft Ez source (:949-951),
//   Ez probes (:956-958).
// The E interior reads only H cells of the interior boxes, so the two
// half-steps are separate launches that update their fields in place.
//
// Layout: (group, z, y, x, L float4), tx innermost.  A block is 128 threads =
// 128/L cells of one x-row; each thread walks a z segment carrying the
// z-neighbour planes in registers.  Per-cell coefficients are float4
// (da, db, ca, cb).
#include "../../include/ceep_b200.h"
#include "common.cuh"
#include "fdtd3d.cuh"

namespace ceep {

constexpr int kThreads3d = 128;

// ---------------------------------------------------------------------------
// H half-step
// ---------------------------------------------------------------------------
// GEN = false for blocks whose cells all lie inside the three H interior
// boxes and off every CPML face: the region tests and face code fold away.
// FACES (bits 1, 2, 4 = x, y, z) selects the CPML face code compiled in:
// a cell outside the box lies on one face (a slab) or on several (an edge or
// corner); the slabs' launches carry only their own face's code.
template <int L, bool GEN, int FACES = 7>
__device__ __forceinline__ void h_segment(const Fdtd3dParams& p, int x, int lo, int y, int g, int z0, int z1) {
  const int nx = p.nx, ny = p.ny, nz = p.nz, n = p.n;
  const size_t gs = (size_t)g * p.gs_field;
  const float4* __restrict__ ex = p.ex + gs;
  const float4* __restrict__ ey = p.ey + gs;
  const float4* __restrict__ ez = p.ez + gs;
  float4* hx = p.hx + gs;
  float4* hy = p.hy + gs;
  float4* hz = p.hz + gs;
  const float4* coef = reinterpret_cast<const float4*>(p.coef);
  const size_t sx = L, sy = (size_t)nx * L, sz = (size_t)ny * nx * L;  // float4 strides
  const float inv = p.inv_dx;
  const bool x_int_hx = x >= n && x < nx - n, x_int = x >= n && x < nx - 1;
  const bool y_int_hy = y >= n && y < ny - n, y_int = y >= n && y < ny - 1;
  const int xf = x < n ? x : (x >= nx - n ? n + (x - (nx - n)) : -1);   // x-face slot
  const int xc = x < n ? x : nx - 1 - x;                                  // its coefficient
  const int yf = y < n ? y : (y >= ny - n ? n + (y - (ny - n)) : -1);
  const int yc = y < n ? y : ny - 1 - y;

  size_t at = (size_t)z0 * sz + (size_t)y * sy + (size_t)x * sx + lo;
  float4 exc = ld4(ex + at), eyc = ld4(ey + at), ezc = ld4(ez + at);
  float4 exm = f4(0.f), eym = f4(0.f);
  if (z0 > 0) { exm = ld4(ex + at - sz); eym = ld4(ey + at - sz); }
  for (int z = z0; z < z1; ++z, at += sz) {
    const bool up = z + 1 < nz;
    const float4 exu = up ? ld4(ex + at + sz) : f4(0.f);
    const float4 eyu = up ? ld4(ey + at + sz) : f4(0.f);
    const float4 ezxp = x + 1 < nx ? ld4(ez + at + sx) : f4(0.f);
    const float4 eyxp = x + 1 < nx ? ld4(ey + at + sx) : f4(0.f);
    const float4 ezyp = y + 1 < ny ? ld4(ez + at + sy) : f4(0.f);
    const float4 exyp = y + 1 < ny ? ld4(ex + at + sy) : f4(0.f);
    const float4 cf = __ldg(coef + (size_t)z * ny * nx + (size_t)y * nx + x);  // da, db, ca, cb
    float4 Hx = hx[at], Hy = hy[at], Hz = hz[at];
    const bool z_int = !GEN || (z >= n && z < nz - 1), z_int_hz = !GEN || (z >= n && z < nz - n);
    // interior boxes (fdtd_3d_batched.py:764-818)
    if (!GEN || (x_int_hx && y_int && z_int))
      Hx = cf.x * Hx + cf.y * ((eyu - eyc) * f4(inv) - (ezyp - ezc) * f4(inv));
    if (!GEN || (x_int && y_int_hy && z_int))
      Hy = cf.x * Hy + cf.y * ((ezxp - ezc) * f4(inv) - (exu - exc) * f4(inv));
    if (!GEN || (x_int && y_int && z_int_hz))
      Hz = cf.x * Hz + cf.y * ((exyp - exc) * f4(inv) - (eyxp - eyc) * f4(inv));
    if (GEN && n > 0) {
      // x faces (:398-460)
      if ((FACES & 1) && xf >= 0) {
        const bool lof = x < n;
        const float4 ezn = lof ? ezxp : ld4(ez + at - sx);
        const float4 eyn = lof ? eyxp : ld4(ey + at - sx);
        const float4 dez = lof ? (ezn - ezc) * f4(inv) : (ezc - ezn) * f4(inv);
        const float4 dey = lof ? (eyn - eyc) * f4(inv) : (eyc - eyn) * f4(inv);
        const size_t pi = (((size_t)z * ny + y) * 2 * n + xf) * L + lo + (size_t)g * p.gs_px;
        const float4 pa = p.cpml_b[xc] * p.psi_hxy[pi] + p.cpml_c[xc] * dez;
        const float4 pb = p.cpml_b[xc] * p.psi_hzy[pi] + p.cpml_c[xc] * dey;
        p.psi_hxy[pi] = pa;
        p.psi_hzy[pi] = pb;
        if (z < nz - 1) Hy = cf.x * Hy - cf.y * pa;
        if (y < ny - 1) Hz = cf.x * Hz + cf.y * pb;
      }
      // y faces (:462-523)
      if ((FACES & 2) && yf >= 0) {
        const bool lof = y < n;
        const float4 ezn = lof ? ezyp : ld4(ez + at - sy);
        const float4 exn = lof ? exyp : ld4(ex + at - sy);
        const float4 dez = lof ? (ezn - ezc) * f4(inv) : (ezc - ezn) * f4(inv);
        const float4 dex = lof ? (exn - exc) * f4(inv) : (exc - exn) * f4(inv);
        const size_t pi = (((size_t)z * 2 * n + yf) * nx + x) * L + lo + (size_t)g * p.gs_py;
        const float4 pa = p.cpml_b[yc] * p.psi_hyx[pi] + p.cpml_c[yc] * dez;
        const float4 pb = p.cpml_b[yc] * p.psi_hzx[pi] + p.cpml_c[yc] * dex;
        p.psi_hyx[pi] = pa;
        p.psi_hzx[pi] = pb;
        if (z < nz - 1) Hx = cf.x * Hx - cf.y * pa;
        if (x < nx - 1) Hz = cf.x * Hz + cf.y * pb;
      }
      // z faces (:525-586)
      const int zf = z < n ? z : (z >= nz - n ? n + (z - (nz - n)) : -1);
      if ((FACES & 4) && zf >= 0) {
        const bool lof = z < n;
        const int zc = lof ? z : nz - 1 - z;
        const float4 dey = lof ? (eyu - eyc) * f4(inv) : (eyc - eym) * f4(inv);
        const float4 dex = lof ? (exu - exc) * f4(inv) : (exc - exm) * f4(inv);
        const size_t pi = (((size_t)zf * ny + y) * nx + x) * L + lo + (size_t)g * p.gs_pz;
        const float4 pa = p.cpml_b[zc] * p.psi_hxz[pi] + p.cpml_c[zc] * dey;
        const float4 pb = p.cpml_b[zc] * p.psi_hyz[pi] + p.cpml_c[zc] * dex;
        p.psi_hxz[pi] = pa;
        p.psi_hyz[pi] = pb;
        if (y < ny - 1) Hx = cf.x * Hx + cf.y * pa;
        if (x < nx - 1) Hy = cf.x * Hy - cf.y * pb;
      }
    }
    hx[at] = Hx;
    hy[at] = Hy;
    hz[at] = Hz;
    exm = exc; eym = eyc;
    exc = exu; eyc = eyu;
    ezc = up ? ld4(ez + at + sz) : f4(0.f);
  }
}

// The H half-step is two launches over disjoint cells.  The box
// [n, N-m)^3 (m = max(n, 1)) lies inside all three interior boxes and on no
// CPML face, so its cells take the lean path (no region tests, no face code,
// fewer registers, more resident warps); the shell around it takes the
// general path.  Both only read E, so their order does not matter.
template <int L>
__global__ void __launch_bounds__(kThreads3d, 8) fdtd3d_h_box_kernel(const Fdtd3dParams p, int zsegs) {
  constexpr int CX = kThreads3d / L;
  const int n = p.n, m = n > 1 ? n : 1;
  const int x = n + blockIdx.x * CX + threadIdx.x / L;
  const int lo = threadIdx.x % L;
  const int y = n + blockIdx.y;
  const int zseg = blockIdx.z % zsegs, g = blockIdx.z / zsegs;
  const int z0 = n + zseg * p.zrows, z1 = min(z0 + p.zrows, p.nz - m);
  if (x >= p.nx - m) return;
  h_segment<L, false>(p, x, lo, y, g, z0, z1);
}

// The shell as lists of cell boxes [x0,x1) x [y0,y1) x [z0,z1), one launch
// per kind of cell: the z slabs, x slabs and y slabs next to the box (cells
// on that one CPML face: FACES = 4, 1, 2) and the edges and corners (every
// face, FACES = 7).  A thread walks at most zr cells of one (x, y) column;
// consecutive threads take consecutive lanes and x (coalesced).
struct ShellBoxes {
  int count;
  int b[12][6];   // x0, x1, y0, y1, z0, z1
};

template <int L, int FACES>
__global__ void __launch_bounds__(kThreads3d, FACES == 7 ? 4 : 6) fdtd3d_h_shell_kernel(const Fdtd3dParams p,
                                                                                          const ShellBoxes sb, int zr) {
  const long long t = (long long)blockIdx.x * kThreads3d + threadIdx.x;
  const int lo = (int)(t % L), g = blockIdx.y;
  long long c = t / L;
  for (int i = 0; i < sb.count; ++i) {
    const int* b = sb.b[i];
    const int w = b[1] - b[0], cols = w * (b[3] - b[2]);
    const long long items = (long long)cols * ((b[5] - b[4] + zr - 1) / zr);
    if (c < items) {
      const int seg = (int)(c / cols), col = (int)(c % cols);
      const int z0 = b[4] + seg * zr;
      h_segment<L, true, FACES>(p, b[0] + col % w, lo, b[2] + col / w, g, z0, min(z0 + zr, b[5]));
      return;
    }
    c -= items;
  }
}

static void add_box(ShellBoxes& sb, int x0, int x1, int y0, int y1, int z0, int z1) {
  if (x0 < x1 && y0 < y1 && z0 < z1) {
    int* b = sb.b[sb.count++];
    b[0] = x0; b[1] = x1; b[2] = y0; b[3] = y1; b[4] = z0; b[5] = z1;
  }
}

static long long shell_items(const ShellBoxes& sb, int zr) {
  long long n = 0;
  for (int i = 0; i < sb.count; ++i) {
    const int* b = sb.b[i];
    n += (long long)(b[1] - b[0]) * (b[3] - b[2]) * ((b[5] - b[4] + zr - 1) / zr);
  }
  return n;
}

template <int L, int FACES>
static cudaError_t launch_shell(const Fdtd3dParams& p, const ShellBoxes& sb, cudaStream_t s) {
  const long long items = shell_items(sb, p.zrows_shell);
  if (items == 0) return cudaSuccess;
  dim3 gs((unsigned)((L * items + kThreads3d - 1) / kThreads3d), p.groups);
  fdtd3d_h_shell_kernel<L, FACES><<<gs, kThreads3d, 0, s>>>(p, sb, p.zrows_shell);
  return cudaGetLastError();
}

// The cells outside the box [n, nx-m) x [n, ny-m) x [n, nz-m) by kind; with
// no box (a grid too small for one) every cell goes to the general list.
template <int L>
static cudaError_t launch_shells(const Fdtd3dParams& p, bool box, cudaStream_t s) {
  const int nx = p.nx, ny = p.ny, nz = p.nz, n = p.n, m = n > 1 ? n : 1;
  ShellBoxes fz{}, fx{}, fy{}, all{};
  if (!box) {
    add_box(all, 0, nx, 0, ny, 0, nz);
    return launch_shell<L, 7>(p, all, s);
  }
  const int xs[2][2] = {{0, n}, {nx - m, nx}}, ys[2][2] = {{0, n}, {ny - m, ny}}, zs[2][2] = {{0, n}, {nz - m, nz}};
  for (int k = 0; k < 2; ++k) {
    add_box(fz, n, nx - m, n, ny - m, zs[k][0], zs[k][1]);          // z slabs
    add_box(fx, xs[k][0], xs[k][1], n, ny - m, n, nz - m);          // x slabs
    add_box(fy, n, nx - m, ys[k][0], ys[k][1], n, nz - m);          // y slabs
    for (int q = 0; q < 2; ++q) add_box(all, xs[k][0], xs[k][1], ys[q][0], ys[q][1], n, nz - m);  // z edges
    add_box(all, 0, nx, 0, n, zs[k][0], zs[k][1]);                    // the z slabs' rims
    add_box(all, 0, nx, ny - m, ny, zs[k][0], zs[k][1]);
    add_box(all, 0, n, n, ny - m, zs[k][0], zs[k][1]);
    add_box(all, nx - m, nx, n, ny - m, zs[k][0], zs[k][1]);
  }
  cudaError_t e;
  if ((e = launch_shell<L, 7>(p, all, s)) != cudaSuccess) return e;
  if ((e = launch_shell<L, 4>(p, fz, s)) != cudaSuccess) return e;
  if ((e = launch_shell<L, 1>(p, fx, s)) != cudaSuccess) return e;
  return launch_shell<L, 2>(p, fy, s);
}

// ---------------------------------------------------------------------------
// E half-step on the interior box, with the Debye/Lorentz currents of each
// component (the 3D analogue of dispersive.py:364-404 / fdtd_2d.py:163-178).
// ---------------------------------------------------------------------------
template <int L, int ND, int NL>
__global__ void __launch_bounds__(kThreads3d, 8) fdtd3d_e_kernel(const Fdtd3dParams p, int step) {
  constexpr int CX = kThreads3d / L;
  constexpr int NP = ND + NL;
  const int n = p.n, nx = p.nx, ny = p.ny, nz = p.nz;
  const int x = n + 1 + blockIdx.x * CX + threadIdx.x / L;
  const int lo = threadIdx.x % L;
  const int y = n + 1 + blockIdx.y;
  const int zseg = blockIdx.z % p.zsegs_e, g = blockIdx.z / p.zsegs_e;
  const int z0 = n + 1 + zseg * p.zrows, z1 = min(z0 + p.zrows, nz - n);
  if (x >= nx - n) return;
  const size_t gs = (size_t)g * p.gs_field;
  float4* ex = p.ex + gs;
  float4* ey = p.ey + gs;
  float4* ez = p.ez + gs;
  const float4* __restrict__ hx = p.hx + gs;
  const float4* __restrict__ hy = p.hy + gs;
  const float4* __restrict__ hz = p.hz + gs;
  const float4* coef = reinterpret_cast<const float4*>(p.coef);
  const float4* ade = reinterpret_cast<const float4*>(p.ade_coef);
  const size_t sx = L, sy = (size_t)nx * L, sz = (size_t)ny * nx * L;
  const size_t cells = (size_t)nx * ny * nz;
  const float inv = p.inv_dx;
  size_t at = (size_t)z0 * sz + (size_t)y * sy + (size_t)x * sx + lo;
  float4 hxm = ld4(hx + at - sz), hym = ld4(hy + at - sz);
  // the save slot covers the interior box only: (G, nzi, nyi, nxi, L)
  const int nxi = nx - 2 * n - 1, nyi = ny - 2 * n - 1, nzi = nz - 2 * n - 1;
  float4* save = p.save_e ? p.save_e + (size_t)(step + 1 - p.save_base) * 3 * p.save_cs +
                                (size_t)g * nzi * nyi * nxi * L +
                                ((size_t)(z0 - n - 1) * nyi + (y - n - 1)) * nxi * L + (size_t)(x - n - 1) * L + lo
                          : nullptr;
  const size_t save_sz = (size_t)nyi * nxi * L;
  for (int z = z0; z < z1; ++z, at += sz) {
    const float4 Hx = ld4(hx + at), Hy = ld4(hy + at), Hz = ld4(hz + at);
    const float4 hzy = ld4(hz + at - sy), hzx = ld4(hz + at - sx);
    const float4 hyx = ld4(hy + at - sx), hxy = ld4(hx + at - sy);
    const size_t cell = (size_t)z * ny * nx + (size_t)y * nx + x;
    const float4 cf = __ldg(coef + cell);
    const float4 cx_ = (Hz - hzy) * f4(inv) - (Hy - hym) * f4(inv);
    const float4 cy_ = (Hx - hxm) * f4(inv) - (Hz - hzx) * f4(inv);
    const float4 cz_ = (Hy - hyx) * f4(inv) - (Hx - hxy) * f4(inv);
    float4* E[3] = {ex + at, ey + at, ez + at};
    const float4 curl[3] = {cx_, cy_, cz_};
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      const float4 e0 = *E[c];
      float4 e = cf.z * e0 + cf.w * curl[c];
      if constexpr (NP > 0) {
        const size_t jbase = (size_t)g * p.gs_j + (size_t)c * cells * L;
        float4 sum = f4(0.f);
        float4 jq[NP > 0 ? NP : 1];
        float4 kq[NP > 0 ? NP : 1];
#pragma unroll
        for (int q = 0; q < NP; ++q) {
          kq[q] = __ldg(ade + q * cells + cell);
          jq[q] = p.j[jbase + (size_t)q * 3 * cells * L + cell * L + lo];
          sum = (q < ND) ? fma4(kq[q].z, jq[q], sum) : sum + jq[q];
        }
        e = e - cf.w * sum;
        const float4 dedt = (e - e0) * f4(p.inv_dt);
#pragma unroll
        for (int q = 0; q < NP; ++q) {
          float4* jp = p.j + jbase + (size_t)q * 3 * cells * L + cell * L + lo;
          if (q < ND) {
            *jp = kq[q].x * jq[q] + kq[q].y * dedt;
          } else {
            float4* jm = p.j_prev + (size_t)g * p.gs_jp + (size_t)c * cells * L + (size_t)(q - ND) * 3 * cells * L +
                         cell * L + lo;
            const float4 jmv = *jm;
            *jp = kq[q].x * jq[q] + kq[q].z * jmv + kq[q].y * dedt;
            *jm = jq[q];
          }
        }
      }
      *E[c] = e;
      if (save) save[c * p.save_cs] = e;
    }
    if (save) save += save_sz;
    hxm = Hx;
    hym = Hy;
  }
}

// ---------------------------------------------------------------------------
// Epilogue: zero the low faces at source cells, add the source, read probes.
// ---------------------------------------------------------------------------
__global__ void fdtd3d_src_probe_kernel(const Fdtd3dParams p, int step) {
  const int L = p.L;
  const size_t sy = (size_t)p.nx * L, sz = (size_t)p.ny * p.nx * L;
  float* ez = reinterpret_cast<float*>(p.ez);
  const float w = p.waveform[step];
  for (int b = threadIdx.x; b < p.ntx; b += blockDim.x) {
    const int sxx = p.src_xyz[3 * b], syy = p.src_xyz[3 * b + 1], szz = p.src_xyz[3 * b + 2];
    const int g = b / (4 * L), lane = b % (4 * L);
    float* e = ez + 4 * ((size_t)g * p.gs_field + (size_t)szz * sz + (size_t)syy * sy + (size_t)sxx * L) + lane;
    if (sxx == 0 || syy == 0 || szz == 0) *e = 0.f;
    *e += w;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < p.ntx * p.nprobe; i += blockDim.x) {
    const int b = i / p.nprobe, q = i % p.nprobe;
    const int pxx = p.prb_xyz[3 * q], pyy = p.prb_xyz[3 * q + 1], pzz = p.prb_xyz[3 * q + 2];
    const int g = b / (4 * L), lane = b % (4 * L);
    p.probes[((size_t)b * p.nprobe + q) * p.nsteps + step] =
        ez[4 * ((size_t)g * p.gs_field + (size_t)pzz * sz + (size_t)pyy * sy + (size_t)pxx * L) + lane];
  }
}

// ---------------------------------------------------------------------------
template <int L, int ND, int NL>
static cudaError_t step_l(const Fdtd3dParams& p, int step, cudaStream_t s, const Fdtd3dSide* side) {
  constexpr int CX = kThreads3d / L;
  const int n = p.n, m = n > 1 ? n : 1;
  const int bx = p.nx - n - m, by = p.ny - n - m, bz = p.nz - n - m;   // the H box
  const int zsb = bz > 0 ? (bz + p.zrows - 1) / p.zrows : 0;
  const bool box = bx > 0 && by > 0 && bz > 0;
  const bool shell = !p.interior_only || !box;
  const bool fork = side != nullptr && box && shell;
  cudaStream_t s2 = fork ? side->stream : s;
  cudaError_t e;
  if (fork) {
    if ((e = cudaEventRecord(side->fork, s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s2, side->fork, 0)) != cudaSuccess) return e;
  }
  if (shell && (e = launch_shells<L>(p, box, s2)) != cudaSuccess) return e;
  if (box) {
    dim3 gb((bx + CX - 1) / CX, by, zsb * p.groups);
    fdtd3d_h_box_kernel<L><<<gb, kThreads3d, 0, s>>>(p, zsb);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  if (fork) {
    if ((e = cudaEventRecord(side->join, s2)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(s, side->join, 0)) != cudaSuccess) return e;
  }
  const int ni = p.nx - 2 * p.n - 1, nj = p.ny - 2 * p.n - 1;
  if (ni > 0 && nj > 0 && p.zsegs_e > 0) {
    dim3 ge((ni + CX - 1) / CX, nj, p.zsegs_e * p.groups);
    fdtd3d_e_kernel<L, ND, NL><<<ge, kThreads3d, 0, s>>>(p, step);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
  }
  fdtd3d_src_probe_kernel<<<1, 256, 0, s>>>(p, step);
  return cudaGetLastError();
}

template <int ND, int NL>
static cudaError_t step_ade(const Fdtd3dParams& p, int step, cudaStream_t s, const Fdtd3dSide* side) {
  switch (p.L) {
    case 1: return step_l<1, ND, NL>(p, step, s, side);
    case 2: return step_l<2, ND, NL>(p, step, s, side);
    case 4: return step_l<4, ND, NL>(p, step, s, side);
    default: return step_l<8, ND, NL>(p, step, s, side);
  }
}

cudaError_t fdtd3d_launch_step(const Fdtd3dParams& p, int step, cudaStream_t s, const Fdtd3dSide* side) {
  switch (p.n_debye * 3 + p.n_lorentz) {
    case 0: return step_ade<0, 0>(p, step, s, side);
    case 1: return step_ade<0, 1>(p, step, s, side);
    case 2: return step_ade<0, 2>(p, step, s, side);
    case 3: return step_ade<1, 0>(p, step, s, side);
    case 4: return step_ade<1, 1>(p, step, s, side);
    case 6: return step_ade<2, 0>(p, step, s, side);
    default: return cudaErrorInvalidValue;
  }
}

}  // namespace ceep

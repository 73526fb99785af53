// Kernels of the fused 2D TMz batched FDTD step (one and two time steps per
// launch, on one grid or on a packed set of phantoms) and their host-side
// configuration and launch, as templates over the lane width L and the ADE
// shape (ND Debye and NL Lorentz poles).  Each fdtd2d_d<ND>l<NL>.cu includes
// this file and instantiates one ADE shape, so the shapes compile in
// parallel; fdtd2d.cu describes the algorithm and dispatches at run time.
#pragma once
// The float4 lane arithmetic of these kernels uses sm_100's paired FP32
// instructions (see common.cuh).
#define CEEP_PAIRED_FP32
#include "../../include/ceep_b200.h"
#include "common.cuh"
#include "fdtd2d.cuh"
#include "tma.cuh"

namespace ceep {

// Ring depth and the resident blocks per SM the registers are budgeted for.
// The consumer holds two slots (its row and the next row's Ez), so kStages - 2
// row slices per block are in flight while it computes.  Measured on the
// 600x600x16 Debye step: 3 stages x 4 blocks/SM 43.2 us, 4 x 3 42.7 us,
// 5 x 2 49.6 us, 6 x 2 52.5 us.
#ifndef CEEP_STAGES
#define CEEP_STAGES 4
#endif
#ifndef CEEP_MIN_BLOCKS
#define CEEP_MIN_BLOCKS 3
#endif
constexpr int kStages = CEEP_STAGES;
constexpr int kMaxRows = 64;                        // rows per block (row masks are 64-bit)
constexpr uint64_t kWaitLimitNs = 1000000000ull;    // default bound of a wait: 1 s

CEEP_D uint64_t wait_limit(const Fdtd2dParams& p) { return p.wait_ns ? p.wait_ns : kWaitLimitNs; }

// One ring slot: the row slices of one row.  PSI = false is the slot of the
// interior-tile kernel, whose blocks touch no CPML strip: its psi slices
// shrink to one unused float4 each.
template <int L, int NP, int NL, bool PSI = true>
struct Stage2d {
  static constexpr int CX = kConsumers / L;
  float4 ez[(CX + 2) * L];   // cells x0-1 .. x0+CX
  float4 hx[CX * L];         // cells x0 .. x0+CX-1
  float4 hy[(CX + 1) * L];   // cells x0-1 .. x0+CX-1
  float4 coef[CX];           // ca, cb, dt/(eps_r eps0), 0
  float4 phx[PSI ? CX * L : 1];        // H psi of the y strips (for Hx), cells x0..
  float4 pey[PSI ? CX * L : 1];        // E psi of the y strips, cells x0..
  float4 phy[PSI ? (CX + 1) * L : 1];  // H psi of the x strips (for Hy), cells x0-1..
  float4 pex[PSI ? CX * L : 1];        // E psi of the x strips, cells x0..
  float4 ade[NP > 0 ? NP * CX : 1];
  float4 j[NP > 0 ? NP * CX * L : 1];
  float4 jp[NL > 0 ? NL * CX * L : 1];
};

template <int L, int NP, int NL>
constexpr size_t stage_smem_bytes() {
  return kStages * sizeof(Stage2d<L, NP, NL>) + 2 * kStages * sizeof(uint64_t);
}

// Ring depth of the one-step kernel's interior blocks: their psi-less slots
// in the shared memory of kStages full slots (more rows in flight).
template <int L, int NP, int NL>
constexpr int interior_stages1() {
  constexpr size_t slot = sizeof(Stage2d<L, NP, NL, false>) + 2 * sizeof(uint64_t);
  constexpr size_t budget = stage_smem_bytes<L, NP, NL>();
  return 7 * slot <= budget ? 7 : 6 * slot <= budget ? 6 : 5 * slot <= budget ? 5 : kStages;
}

// Slot index and phase parity of a position in an NS-slot mbarrier ring.
template <int NS>
struct RingPos {
  int slot;
  uint32_t phase;
  CEEP_D void advance() {
    if (++slot == NS) {
      slot = 0;
      phase ^= 1u;
    }
  }
};

// Strip bookkeeping shared by producer and consumers.
struct Strips {
  int n, nx, ny;
  // H psi of the y strips (Hx): row -> strip row, or -1
  __device__ int hy_row(int y) const {
    if (y < n) return y;
    if (y >= ny - n && y < ny - 1) return n + (y - (ny - n));
    return -1;
  }
  // E psi of the y strips: row -> strip row, or -1 (rows 1..n and ny-n..ny-1)
  __device__ int ey_row(int y) const {
    if (y >= 1 && y <= n) return y - 1;
    if (n > 0 && y >= ny - n) return n + (y - (ny - n));
    return -1;
  }
};

// ------------------------------------------------------------------------
// Per-cell updates, shared by the one-step and two-step consumers so both run
// the same arithmetic.  GEN = false for blocks entirely inside every region's
// plain interior: the region predicates fold away.  `psi` holds the cell's
// old psi on entry and its new psi on return; `strip` says whether the cell
// is in a strip (then the caller stores psi).
// ------------------------------------------------------------------------
template <bool GEN>
CEEP_D float4 hx_step(const Fdtd2dParams& p, int x, int y, float4 hx, float4 ez_c, float4 ez_up, float4& psi,
                      bool& strip) {
  strip = false;
  const int n = p.n;
  if (!GEN) return fma4(-p.db_dx, ez_up - ez_c, hx);
  if (y >= p.ny - 1) return hx;  // never updated
  const float4 d = ez_up - ez_c;
  if (x >= n && x < p.nx - n && y >= n) hx = fma4(-p.db_dx, d, hx);
  int ci = -1;
  if (y < n) ci = y;
  else if (y >= p.ny - n) ci = p.ny - 1 - y;
  if (ci >= 0) {
    psi = p.cpml_b[ci] * psi + p.cpml_c[ci] * (d * f4(p.inv_dx));
    strip = true;
    hx = fma4(-p.db, psi, hx);
  }
  return hx;
}

template <bool GEN>
CEEP_D float4 hy_step(const Fdtd2dParams& p, int x, int y, float4 hy, float4 ez_c, float4 ez_r, float4& psi,
                      bool& strip) {
  strip = false;
  const int n = p.n;
  if (!GEN) return fma4(p.db_dx, ez_r - ez_c, hy);
  if (x >= p.nx - 1) return hy;  // never updated
  const float4 d = ez_r - ez_c;
  if (x >= n && y >= n && y < p.ny - n) hy = fma4(p.db_dx, d, hy);
  int ci = -1;
  if (x < n) ci = x;
  else if (x >= p.nx - n) ci = p.nx - 1 - x;
  if (ci >= 0) {
    psi = p.cpml_b[ci] * psi + p.cpml_c[ci] * (d * f4(p.inv_dx));
    strip = true;
    hy = fma4(p.db, psi, hy);
  }
  return hy;
}

// As hx_step/hy_step, storing the new psi of a strip cell to `psi_out` (if set).
template <bool GEN>
CEEP_D float4 hx_new(const Fdtd2dParams& p, float4 psi, float4* psi_out, int x, int y, float4 hx, float4 ez_c,
                     float4 ez_up) {
  bool strip;
  const float4 h = hx_step<GEN>(p, x, y, hx, ez_c, ez_up, psi, strip);
  if (strip && psi_out) st4(psi_out, psi);
  return h;
}

template <bool GEN>
CEEP_D float4 hy_new(const Fdtd2dParams& p, float4 psi, float4* psi_out, int x, int y, float4 hy, float4 ez_c,
                     float4 ez_r) {
  bool strip;
  const float4 h = hy_step<GEN>(p, x, y, hy, ez_c, ez_r, psi, strip);
  if (strip && psi_out) st4(psi_out, psi);
  return h;
}

constexpr uint32_t kF9 = 1, kEX = 2, kEY = 4;

// E update of one cell: the interior (ca, cb) update with the Debye/Lorentz
// currents, or the E-CPML strip terms, then edge zeroing.  jq (in J^n, out
// J^{n+1}), jm (Lorentz: in J^{n-1}, out J^n) and pex/pey (strip psi) are
// updated in place; the returned flags say which the caller must store
// (kF9: the currents, kEX / kEY: the x / y strip psi).
//   ADE (dispersive.py:364-404, fdtd_2d.py:163-178):
//     E -= cb * sum(gamma_p J_p);  Debye J = k1 J + k2 dE/dt;
//     Lorentz J' = k1 J + k3 J_prev + k2 dE/dt, J_prev = J
//   E-CPML (fdtd_2d_batched.py:355-406): x strips E += dt/eps * psi_x,
//     y strips E -= dt/eps * psi_y, with no ca factor.
template <bool GEN, int ND, int NL>
CEEP_D float4 e_step(const Fdtd2dParams& p, int x, int y, float4 e, float4 dhy, float4 dhx, float4 cf,
                     const float4* kq, float4* jq, float4* jm, float4& pex, float4& pey, uint32_t& flags) {
  constexpr int NP = ND + NL;
  const int n = p.n, nx = p.nx, ny = p.ny;
  flags = 0;
  const bool f9 = !GEN || (x >= n + 1 && x < nx - n && y >= n + 1 && y < ny - n);
  if (f9) {
    flags |= kF9;
    float4 en = cf.x * e + cf.y * (dhy * f4(p.inv_dx) - dhx * f4(p.inv_dx));
    if constexpr (NP > 0) {
      float4 sum = f4(0.f);
#pragma unroll
      for (int q = 0; q < NP; ++q) sum = (q < ND) ? fma4(kq[q].z, jq[q], sum) : sum + jq[q];
      en = en - cf.y * sum;
      const float4 dedt = (en - e) * f4(p.inv_dt);
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        if (q < ND) {
          jq[q] = kq[q].x * jq[q] + kq[q].y * dedt;
        } else {
          const float4 jold = jq[q];
          jq[q] = kq[q].x * jold + kq[q].z * jm[q - ND] + kq[q].y * dedt;
          jm[q - ND] = jold;
        }
      }
    }
    e = en;
  }
  if (GEN && n > 0) {
    const int ex_s = (x >= 1 && x <= n) ? x - 1 : (x >= nx - n) ? n + (x - (nx - n)) : -1;
    if (y >= 1 && ex_s >= 0) {
      const int ex_c = (x >= 1 && x <= n) ? x - 1 : nx - 1 - x;
      pex = p.cpml_b[ex_c] * pex + p.cpml_c[ex_c] * (dhy * f4(p.inv_dx));
      flags |= kEX;
      e = fma4(cf.z, pex, e);
    }
    const int sey = Strips{n, nx, ny}.ey_row(y);
    if (x >= 1 && sey >= 0) {
      const int ci = (y <= n) ? y - 1 : ny - 1 - y;
      pey = p.cpml_b[ci] * pey + p.cpml_c[ci] * (dhx * f4(p.inv_dx));
      flags |= kEY;
      e = fma4(-cf.z, pey, e);
    }
  }
  if (GEN && (x == 0 || x == nx - 1 || y == 0 || y == ny - 1)) e = f4(0.f);
  return e;
}

// Slots of the adjoint's saved Ez and J for the state after step `step_after`
// (slot step_after - save_base of (slots, G, ...) arrays), at TX group g.
CEEP_D float4* save_ez_slot(const Fdtd2dParams& p, int step_after, int g) {
  return p.save_ez + (size_t)(step_after - p.save_base) * p.groups * p.gs_field + (size_t)g * p.gs_field;
}
CEEP_D float4* save_j_slot(const Fdtd2dParams& p, int step_after, int g) {
  return p.save_j + (size_t)(step_after - p.save_base) * p.groups * p.gs_j + (size_t)g * p.gs_j;
}

// Soft source of `step` (fdtd_2d_batched.py:509-515): the transmit events of
// lane group lane_g whose source is cell (x, y).
CEEP_D void add_sources(const Fdtd2dParams& p, float4& e, int x, int y, int lane_g, int step) {
  const float w = __ldg(p.waveform + step);
  for (int s = 4 * lane_g; s < 4 * lane_g + 4 && s < p.ntx; ++s)
    if (__ldg(p.src_xy + 2 * s) == x && __ldg(p.src_xy + 2 * s + 1) == y) add_comp(e, s & 3, w);
}

// Probe record of `step` (fdtd_2d_batched.py:517-526) for the probes at (x, y).
CEEP_D void record_probes(const Fdtd2dParams& p, float4 e, int x, int y, int lane_g, int step) {
  for (int q = 0; q < p.nprobe; ++q) {
    if (__ldg(p.prb_xy + 2 * q) == x && __ldg(p.prb_xy + 2 * q + 1) == y) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int tx = 4 * lane_g + c;
        if (tx < p.ntx) p.probes[((size_t)tx * p.nprobe + q) * p.nsteps + step] = comp(e, c);
      }
    }
  }
}

// ------------------------------------------------------------------------
// Producer: one thread, bulk copies of row slices into the stage ring.
// ------------------------------------------------------------------------
template <int L, int ND, int NL, int NS = kStages, bool PSI = true>
CEEP_D void produce(const Fdtd2dParams& p, Stage2d<L, ND + NL, NL, PSI>* st, uint64_t* full, uint64_t* empty,
                    int par, int x0, int y0, int y1, int rs, int nslots, int g) {
  constexpr int NP = ND + NL;
  constexpr int CX = kConsumers / L;
  const int nx = p.nx, ny = p.ny, n = p.n;
  const Strips sp{n, nx, ny};
  const size_t gf = (size_t)g * p.gs_field;
  const float4* ez = p.ez[par] + gf;
  const float4* hx = p.hx[par] + gf;
  const float4* hy = p.hy[par] + gf;
  const float4* coef = reinterpret_cast<const float4*>(p.coef);
  const float4* ade = reinterpret_cast<const float4*>(p.ade_coef);
  const float4* J = p.j[par] + (size_t)g * p.gs_j;
  const float4* Jp = p.j_prev[par] + (size_t)g * p.gs_jp;
  const float4* psi_hx = p.psi_hx[par] + (size_t)g * p.gs_psi_y;
  const float4* psi_hy = p.psi_hy[par] + (size_t)g * p.gs_psi_x;
  const float4* psi_ezx = p.psi_ezx[par] + (size_t)g * p.gs_psi_x;
  const float4* psi_ezy = p.psi_ezy[par] + (size_t)g * p.gs_psi_y;
  const size_t plane = (size_t)nx * ny;
  // x0 may be -1 (the first tile of the two-step kernel): cells below 0 are
  // not copied and their slots are never read.
  const int xa = x0 > 0 ? x0 - 1 : 0;                  // first halo cell
  const int xs = x0 > 0 ? x0 : 0;                      // first owned cell
  const int xb = x0 + CX + 1 < nx ? x0 + CX + 1 : nx;  // end of the Ez slice
  const int xe = x0 + CX < nx ? x0 + CX : nx;          // end of the owned cells
  const uint32_t cb = L * 16;                           // bytes of one cell's float4s
  // x-strip cell ranges of this block (empty when lo >= hi)
  const int hl0 = xa, hl1 = min(xe, n);                                  // H, left  (sx = x)
  const int hr0 = max(xa, nx - n), hr1 = min(xe, nx - 1);                // H, right (sx = n + x - (nx-n))
  const int el0 = max(x0, 1), el1 = min(xe, n + 1);                      // E, left  (sx = x - 1)
  const int er0 = max(x0, nx - n), er1 = xe;                             // E, right
  int issued = 0;
  for (int k = 0; k < nslots; ++k) {
    const int s = k % NS, u = k / NS;
    if (u > 0 && !mbar_wait_bounded(&empty[s], (u - 1) & 1, wait_limit(p))) {
      record_status(p.status, CEEP_ERR_TIMEOUT);
      break;
    }
    const int r = rs + k;
    if (r == p.fault_row) {  // injected fault: this slot never fills
      issued = k + 1;
      continue;
    }
    const bool pro = r < y0, tail = r >= y1, body = !pro && !tail;
    const int shy = sp.hy_row(r), sey = sp.ey_row(r);
    Stage2d<L, NP, NL, PSI>& S = st[s];
    const size_t rowc = (size_t)r * nx;
    const size_t rowp = (size_t)r * 2 * n;
    // Two passes over the same list: count the bytes, then issue the copies.
    for (int pass = 0; pass < 2; ++pass) {
      uint32_t bytes = 0;
      auto cp = [&](void* dst, const void* src, uint32_t nb) {
        if (nb == 0) return;
        if (pass) bulk_g2s(dst, src, nb, &full[s]);
        else bytes += nb;
      };
      cp(S.ez + (xa - (x0 - 1)) * L, ez + (rowc + xa) * L, (xb - xa) * cb);
      if (!tail) {
        cp(S.hx + (xs - x0) * L, hx + (rowc + xs) * L, (xe - xs) * cb);
        if (PSI && shy >= 0) cp(S.phx + (xs - x0) * L, psi_hx + ((size_t)shy * nx + xs) * L, (xe - xs) * cb);
      }
      if (body) {
        cp(S.hy + (xa - (x0 - 1)) * L, hy + (rowc + xa) * L, (xe - xa) * cb);
        cp(S.coef + (xs - x0), coef + rowc + xs, (xe - xs) * 16u);
        if (PSI && sey >= 0) cp(S.pey + (xs - x0) * L, psi_ezy + ((size_t)sey * nx + xs) * L, (xe - xs) * cb);
        if (PSI && hl1 > hl0) cp(S.phy + (hl0 - (x0 - 1)) * L, psi_hy + (rowp + hl0) * L, (hl1 - hl0) * cb);
        if (PSI && hr1 > hr0) cp(S.phy + (hr0 - (x0 - 1)) * L, psi_hy + (rowp + n + hr0 - (nx - n)) * L, (hr1 - hr0) * cb);
        if (PSI && el1 > el0) cp(S.pex + (el0 - x0) * L, psi_ezx + (rowp + el0 - 1) * L, (el1 - el0) * cb);
        if (PSI && er1 > er0) cp(S.pex + (er0 - x0) * L, psi_ezx + (rowp + n + er0 - (nx - n)) * L, (er1 - er0) * cb);
#pragma unroll
        for (int q = 0; q < NP; ++q) {
          cp(S.ade + q * CX + (xs - x0), ade + q * plane + rowc + xs, (xe - xs) * 16u);
          cp(S.j + (q * CX + xs - x0) * L, J + (q * plane + rowc + xs) * L, (xe - xs) * cb);
        }
#pragma unroll
        for (int q = 0; q < NL; ++q)
          cp(S.jp + (q * CX + xs - x0) * L, Jp + (q * plane + rowc + xs) * L, (xe - xs) * cb);
      }
      if (!pass) mbar_arrive_expect_tx(&full[s], bytes);
    }
    issued = k + 1;
  }
  // Let every copy this thread issued land before it leaves (only matters on
  // the timeout path: otherwise the consumers have waited on all of them).
  for (int k = issued > NS ? issued - NS : 0; k < issued; ++k)
    mbar_wait_bounded(&full[k % NS], (k / NS) & 1, wait_limit(p));
}

// ------------------------------------------------------------------------
// Consumer: one float4 (4 TX) of one cell per thread, walking the rows.
// ------------------------------------------------------------------------
template <int L, bool GEN, int ND, int NL, bool PSI = true, int NS = kStages>
CEEP_D void consume(const Fdtd2dParams& p, Stage2d<L, ND + NL, NL, PSI>* st, uint64_t* full, uint64_t* empty,
                    int step, int par, int x0, int y0, int y1, int rs, int nslots, int g) {
  static_assert(PSI || !GEN, "the general path reads the staged psi slices");
  constexpr int NP = ND + NL;
  constexpr int CX = kConsumers / L;
  const int nx = p.nx, ny = p.ny, n = p.n;
  const Strips sp{n, nx, ny};
  const int cx = threadIdx.x / L, lo = threadIdx.x % L;
  const int x = x0 + cx;
  const bool active = x < nx;
  const int lane_warp = threadIdx.x & 31;
  const size_t gf = (size_t)g * p.gs_field;
  float4* ezw = p.ez[par ^ 1] + gf;
  float4* hxw = p.hx[par ^ 1] + gf;
  float4* hyw = p.hy[par ^ 1] + gf;
  float4* psi_hx_out = p.psi_hx[par ^ 1] + (size_t)g * p.gs_psi_y;
  float4* psi_hy_out = p.psi_hy[par ^ 1] + (size_t)g * p.gs_psi_x;
  float4* psi_ezx = p.psi_ezx[par ^ 1] + (size_t)g * p.gs_psi_x;
  float4* psi_ezy = p.psi_ezy[par ^ 1] + (size_t)g * p.gs_psi_y;
  float4* J = p.j[par ^ 1] + (size_t)g * p.gs_j;
  float4* Jp = p.j_prev[par ^ 1] + (size_t)g * p.gs_jp;
  const size_t plane = (size_t)nx * ny;
  const int lane_g = g * L + lo;  // float4 lane across all groups (tx = 4*lane_g + c)
  // x-strip membership of this cell (H: Hy at x and x-1; E: Ez at x)
  const int hxs = (x < n) ? x : (x >= nx - n && x < nx - 1) ? n + (x - (nx - n)) : -1;
  const int ex_s = (x >= 1 && x <= n) ? x - 1 : (x >= nx - n) ? n + (x - (nx - n)) : -1;

  // Source/probe rows of this segment as bit masks (rows <= 64).
  uint64_t src_rows = 0, prb_rows = 0;
  for (int y = y0; y < y1; ++y) {
    const uint8_t f = __ldg(p.row_flags + y);
    if (f & 1) src_rows |= 1ull << (y - y0);
    if (f & 2) prb_rows |= 1ull << (y - y0);
  }

  // Warp-uniform bounded wait: if any lane gives up, the whole warp leaves.
  auto wait = [&](RingPos<NS> c) {
    const bool ok = mbar_wait_bounded(&full[c.slot], c.phase, wait_limit(p));
    if (__any_sync(0xffffffffu, !ok)) {
      if (lane_warp == 0) record_status(p.status, CEEP_ERR_TIMEOUT);
      return false;
    }
    return true;
  };
  auto release = [&](int slot) {
    __syncwarp();
    if (lane_warp == 0) mbar_arrive(&empty[slot]);
  };

  // ring position of slice k+1 and the slot of slice k (k from 0 at row rs)
  RingPos<NS> up{0, 0u};
  int cs = 0;
  if (!wait(up)) return;
  up.advance();
  int k = 0;
  float4 hx_prev = f4(0.f);
  if (y0 > 0) {  // slot 0 holds row y0-1 (Ez, Hx, H psi): Hx^{n+1/2}(x, y0-1)
    if (!wait(up)) return;
    if (active) {
      const Stage2d<L, NP, NL, PSI>& A = st[0];
      hx_prev = hx_new<GEN>(p, GEN ? A.phx[cx * L + lo] : f4(0.f), nullptr, x, y0 - 1, A.hx[cx * L + lo],
                            A.ez[(cx + 1) * L + lo], st[up.slot].ez[(cx + 1) * L + lo]);
    }
    release(cs);
    cs = up.slot;
    up.advance();
    k = 1;
  }

  for (int y = y0; y < y1; ++y, ++k) {
    const bool has_up = k + 1 < nslots;
    if (has_up && !wait(up)) return;
    const Stage2d<L, NP, NL, PSI>& A = st[cs];
    if (active) {
      const int i0 = (cx + 1) * L + lo;  // this cell in the halo'd slices
      const float4 ez_c = A.ez[i0];
      const float4 ez_up = has_up ? st[up.slot].ez[i0] : f4(0.f);
      const size_t at = ((size_t)y * nx + x) * L + lo;
      const int shy = GEN ? sp.hy_row(y) : -1;
      const int sey = GEN ? sp.ey_row(y) : -1;

      // H phase: this cell, plus the recomputed Hy of the left neighbour
      const float4 hxn = hx_new<GEN>(p, GEN ? A.phx[cx * L + lo] : f4(0.f),
                                     shy >= 0 ? psi_hx_out + ((size_t)shy * nx + x) * L + lo : nullptr, x, y,
                                     A.hx[cx * L + lo], ez_c, ez_up);
      const float4 hyn = hy_new<GEN>(p, GEN ? A.phy[i0] : f4(0.f), hxs >= 0 ? psi_hy_out + ((size_t)y * 2 * n + hxs) * L + lo : nullptr,
                                     x, y, A.hy[i0], ez_c, A.ez[i0 + L]);
      float4 hyl = f4(0.f);
      if (!GEN || x >= 1)
        hyl = hy_new<GEN>(p, GEN ? A.phy[i0 - L] : f4(0.f), nullptr, x - 1, y, A.hy[i0 - L], A.ez[i0 - L], ez_c);
      st4(hxw + at, hxn);
      st4(hyw + at, hyn);

      // E phase
      constexpr int NQ = NP > 0 ? NP : 1, NLQ = NL > 0 ? NL : 1;
      float4 kq[NQ], jq[NQ], jm[NLQ];
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        kq[q] = A.ade[q * CX + cx];
        jq[q] = A.j[(q * CX + cx) * L + lo];
      }
#pragma unroll
      for (int q = 0; q < NL; ++q) jm[q] = A.jp[(q * CX + cx) * L + lo];
      float4 pex = GEN ? A.pex[cx * L + lo] : f4(0.f), pey = GEN ? A.pey[cx * L + lo] : f4(0.f);
      uint32_t fl;
      float4 e = e_step<GEN, ND, NL>(p, x, y, ez_c, hyn - hyl, hxn - hx_prev, A.coef[cx], kq, jq, jm, pex, pey, fl);
      if (NP > 0 && (fl & kF9)) {
#pragma unroll
        for (int q = 0; q < NP; ++q) {
          const size_t ja = (q * plane + (size_t)y * nx + x) * L + lo;
          st4(J + ja, jq[q]);
          if (q < ND && p.save_j)
            st4(p.save_j + (size_t)(step + 1 - p.save_base) * p.groups * p.gs_j + (size_t)g * p.gs_j + ja, jq[q]);
        }
#pragma unroll
        for (int q = 0; q < NL; ++q) st4(Jp + (q * plane + (size_t)y * nx + x) * L + lo, jm[q]);
      }
      if (fl & kEX) st4(psi_ezx + ((size_t)y * 2 * n + ex_s) * L + lo, pex);
      if (fl & kEY) st4(psi_ezy + ((size_t)sey * nx + x) * L + lo, pey);

      // soft source and probe record (fdtd_2d_batched.py:509-526)
      if ((src_rows >> (y - y0)) & 1) add_sources(p, e, x, y, lane_g, step);
      if ((prb_rows >> (y - y0)) & 1) record_probes(p, e, x, y, lane_g, step);
      st4(ezw + at, e);
      if (p.save_ez) st4(p.save_ez + (size_t)(step + 1 - p.save_base) * p.groups * p.gs_field + gf + at, e);
      hx_prev = hxn;
    }
    release(cs);
    cs = up.slot;
    up.advance();
  }
  if (k < nslots) release(cs);  // the Ez-only slot of row y1
}

// One block's work for one time step with ring slots of one kind: PSI (a
// frame block: kStages full slots, the general code) or not (an interior
// block: NS psi-less slots in the same shared memory, the interior code).
template <int L, int ND, int NL, bool PSI, int NS>
CEEP_D void step_run(const Fdtd2dParams& p, int step, int par, int x0, int y0, int y1, int g,
                     unsigned char* smem_raw) {
  using St = Stage2d<L, ND + NL, NL, PSI>;
  St* st = reinterpret_cast<St*>(smem_raw);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NS * sizeof(St));
  uint64_t* empty = full + NS;
  const int rs = y0 > 0 ? y0 - 1 : 0;
  const int nslots = (y1 - rs) + (y1 < p.ny ? 1 : 0);

  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumers / 32);
    }
    mbar_init_fence();
  }
  __syncthreads();
  // Programmatic dependent launch: let the next step's blocks be scheduled as
  // this grid drains, and wait for the previous step's grid to finish (and
  // its writes to be visible) before touching any field.  Every global read
  // and write of field state comes after the wait, which also protects the
  // ping-pong buffer the previous step was still reading.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");

  if (threadIdx.x >= kConsumers) {
    if (threadIdx.x == kConsumers) produce<L, ND, NL, NS, PSI>(p, st, full, empty, par, x0, y0, y1, rs, nslots, g);
    return;
  }
  consume<L, PSI, ND, NL, PSI, NS>(p, st, full, empty, step, par, x0, y0, y1, rs, nslots, g);
}

// One block's work for one time step: a column strip of CX cells starting at
// x0, rows [y0, y0 + rows), TX group g.  Shared by the single-grid kernel and
// the packed multi-phantom kernel.  Block-uniform: every owned cell (and every
// recomputed halo H) lies in the plain interior of all regions; the far
// column/row is excluded too (Hy(nx-1), Hx(ny-1) are never updated and Ez
// there is an edge).
template <int L, int ND, int NL>
CEEP_D void step_block(const Fdtd2dParams& p, int step, int par, int x0, int y0, int g, unsigned char* smem_raw) {
  constexpr int CX = kConsumers / L;
  const int y1 = min(y0 + p.rows, p.ny);
  const int n = p.n, m = n > 1 ? n : 1;
  const bool interior = (x0 >= n + 1) && (x0 + CX <= p.nx - m) && (y0 >= n + 1) && (y1 <= p.ny - m);
  constexpr int NSI = interior_stages1<L, ND + NL, NL>();
  static_assert(NSI * (sizeof(Stage2d<L, ND + NL, NL, false>) + 2 * sizeof(uint64_t)) <=
                    stage_smem_bytes<L, ND + NL, NL>(),
                "interior slots must fit the general blocks' shared memory");
  if (interior)
    step_run<L, ND, NL, false, NSI>(p, step, par, x0, y0, y1, g, smem_raw);
  else
    step_run<L, ND, NL, true, kStages>(p, step, par, x0, y0, y1, g, smem_raw);
}

template <int L, int ND, int NL>
__global__ void __launch_bounds__(kConsumers + 32, CEEP_MIN_BLOCKS) fdtd2d_step_kernel(const Fdtd2dParams p, int step, int par) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int CX = kConsumers / L;
  int bx, by;
  tile_frame_first(blockIdx.x, (p.nx + CX - 1) / CX, (p.ny + p.rows - 1) / p.rows, p.frame1[0], p.frame1[1],
                   p.frame1[2], p.frame1[3], bx, by);
  step_block<L, ND, NL>(p, step, par, bx * CX, by * p.rows, blockIdx.z, smem_raw);
}

// ------------------------------------------------------------------------
// Two steps per launch (temporal block of two).  The block's 128/L thread
// columns start one column left of its output columns: step A (n -> n+1)
// runs, exactly as the one-step consumer, on all CX columns and on the rows
// ya0 = y0-1 .. ya1-1 = y1 (one row of halo each side), keeping its results
// on chip; step B (n+1 -> n+2) runs one row behind A on the inner CX-2
// columns and the rows [y0, y1) and is the only one that writes HBM.  B reads
// A's E^{n+1}, Hy^{n+1/2} and x-strip H psi of the neighbouring columns
// through a two-row shared-memory exchange; everything else B needs from A is
// its own column's, kept in registers.  One iteration runs A on row r and B
// on row r-1 (independent work for the scheduler) and ends with the one
// consumer barrier of the row, which orders A's exchange writes of row r
// before B's reads of it in the next iteration and B's reads of row r-1
// before A overwrites that buffer with row r+1.  Each state word is read once
// and written once per two steps.
// ------------------------------------------------------------------------
// Ring slots of the two-step kernel: a frame block has kStages2 full slots
// (three leave shared memory for three blocks per SM); an interior block
// lays the same shared memory out as interior_stages2() psi-less slots, so
// more of its rows are in flight.
#ifndef CEEP_STAGES2
#define CEEP_STAGES2 3
#endif
constexpr int kStages2 = CEEP_STAGES2;
#ifndef CEEP_MIN_BLOCKS2I
#define CEEP_MIN_BLOCKS2I 4  // the interior-tile kernel (one or no ADE pole)
#endif
#ifndef CEEP_MIN_BLOCKS2
#define CEEP_MIN_BLOCKS2 3
#endif

template <int L>
struct Exch2 {
  float4 e[kConsumers];    // E^{n+1}
  float4 hy[kConsumers];   // Hy^{n+1/2}
  float4 phy[kConsumers];  // x-strip psi of Hy after step A
};

// Bytes of a two-step block's shared memory with NS ring slots of the given kind.
template <int L, int ND, int NL, bool PSI, int NS>
constexpr size_t step2_layout_bytes() {
  return NS * sizeof(Stage2d<L, ND + NL, NL, PSI>) + 2 * NS * sizeof(uint64_t) + 2 * sizeof(Exch2<L>) + 16;
}

// Ring depth of interior blocks: their slots carry no psi slices, so the
// shared memory of the general blocks' kStages2 full slots holds four or
// five of theirs (more rows in flight ahead of the consumers).
template <int L, int ND, int NL>
constexpr int interior_stages2() {
  constexpr size_t budget = step2_layout_bytes<L, ND, NL, true, kStages2>();
  return step2_layout_bytes<L, ND, NL, false, 5>() <= budget   ? 5
         : step2_layout_bytes<L, ND, NL, false, 4>() <= budget ? 4
                                                               : kStages2;
}

// Dynamic shared memory of the two-step kernel (PSI: any block may be a
// frame block) and of the interior-tile kernel (PSI = false).
template <int L, int ND, int NL, bool PSI = true>
constexpr size_t step2_smem_bytes() {
  return PSI ? step2_layout_bytes<L, ND, NL, true, kStages2>()
             : step2_layout_bytes<L, ND, NL, false, interior_stages2<L, ND, NL>()>();
}

CEEP_D void consumer_barrier() { asm volatile("bar.sync 1, %0;" ::"n"(kConsumers) : "memory"); }

// RR = false: a block none of whose rows holds a source or a probe, in a run
// that saves nothing for the adjoint (the loop compiles without those paths).
template <int L, bool GEN, int ND, int NL, bool PK, bool PSI = true, bool RR = true, int NS = kStages2>
CEEP_D void consume2(const Fdtd2dParams& p, Stage2d<L, ND + NL, NL, PSI>* st, uint64_t* full, uint64_t* empty,
                     Exch2<L>* xr, volatile int* abort_flag, int step, int par, int x0, int y0, int y1, int ya0,
                     int ya1, int rs, int nslots, int g) {
  static_assert(PSI || !GEN, "the general path reads the staged psi slices");
  constexpr int NP = ND + NL, NQ = NP > 0 ? NP : 1, NLQ = NL > 0 ? NL : 1;
  constexpr int CX = kConsumers / L;
  const int nx = p.nx, ny = p.ny, n = p.n;
  const Strips sp{n, nx, ny};
  const int t = threadIdx.x, cx = t / L, lo = t % L;
  const int x = x0 + cx;
  const bool valid = x >= 0 && x < nx;                  // step A computes this column
  const bool own = valid && cx >= 1 && cx < CX - 1;     // step B computes and writes it
  const int lane_warp = t & 31, lane_g = g * L + lo;
  const size_t gf = (size_t)g * p.gs_field, plane = (size_t)nx * ny;
  float4* ezw = p.ez[par ^ 1] + gf;
  float4* hxw = p.hx[par ^ 1] + gf;
  float4* hyw = p.hy[par ^ 1] + gf;
  float4* psi_hx_out = p.psi_hx[par ^ 1] + (size_t)g * p.gs_psi_y;
  float4* psi_hy_out = p.psi_hy[par ^ 1] + (size_t)g * p.gs_psi_x;
  float4* psi_ezx = p.psi_ezx[par ^ 1] + (size_t)g * p.gs_psi_x;
  float4* psi_ezy = p.psi_ezy[par ^ 1] + (size_t)g * p.gs_psi_y;
  float4* J = p.j[par ^ 1] + (size_t)g * p.gs_j;
  float4* Jp = p.j_prev[par ^ 1] + (size_t)g * p.gs_jp;
  const int hxs = (x < n) ? x : (x >= nx - n && x < nx - 1) ? n + (x - (nx - n)) : -1;
  const int ex_s = (x >= 1 && x <= n) ? x - 1 : (x >= nx - n) ? n + (x - (nx - n)) : -1;

  // source/probe rows among A's rows [ya0, ya1) (<= 64) as bit masks
  uint64_t src_rows = 0, prb_rows = 0;
  for (int y = ya0; RR && y < ya1; ++y) {
    const uint8_t f = __ldg(p.row_flags + y);
    if (f & 1) src_rows |= 1ull << (y - ya0);
    if (f & 2) prb_rows |= 1ull << (y - ya0);
  }

  // A timed-out wait sets the block's abort flag; the warps then skip every
  // later wait and all arithmetic but keep taking the consumer barrier, so
  // all four reach it the same number of times.
  // Ring positions advance by one slot per row (slot index and phase carried,
  // no division by the ring depth).
  bool aborted = false;
  auto wait = [&](RingPos<NS> c) {
    if (aborted) return;
    const bool ok = mbar_wait_bounded(&full[c.slot], c.phase, wait_limit(p));
    if (__any_sync(0xffffffffu, !ok)) {
      if (lane_warp == 0) {
        record_status(p.status, CEEP_ERR_TIMEOUT);
        *abort_flag = 1;
      }
      aborted = true;
    }
  };
  auto release = [&](int slot) {
    __syncwarp();
    if (lane_warp == 0) mbar_arrive(&empty[slot]);
  };

  // step A's results for this column's previous row, which step B uses next
  float4 pv_hx = f4(0.f), pv_cf = f4(0.f), pv_phx = f4(0.f), pv_pex = f4(0.f), pv_pey = f4(0.f);
  float4 pv_kq[NQ], pv_jq[NQ], pv_jm[NLQ];
#pragma unroll
  for (int q = 0; q < NQ; ++q) pv_kq[q] = pv_jq[q] = f4(0.f);
#pragma unroll
  for (int q = 0; q < NLQ; ++q) pv_jm[q] = f4(0.f);
  float4 hxa_prev = f4(0.f);  // Hx^{n+1/2}(x, r-1)
  float4 hxb_prev = f4(0.f);  // Hx^{n+3/2}(x, y-1)

  // Step B on own row y, given A's E^{n+1}(x, y+1) (zero above the grid).
  auto b_row = [&](int y, float4 e1_up, bool src_row, bool prb_row) {
    const Exch2<L>& XB = xr[y & 1];
    const float4 e1_c = XB.e[t], e1_r = XB.e[t + L], e1_l = XB.e[t - L];
    float4 phy_c = XB.phy[t], phy_l = XB.phy[t - L];
    const size_t at = ((size_t)y * nx + x) * L + lo;
    bool sx, sy2, dummy;
    float4 phx = pv_phx;
    const float4 hxb = hx_step<GEN>(p, x, y, pv_hx, e1_c, e1_up, phx, sx);
    const float4 hyb = hy_step<GEN>(p, x, y, XB.hy[t], e1_c, e1_r, phy_c, sy2);
    float4 hybl = f4(0.f);
    if (!GEN || x >= 1) hybl = hy_step<GEN>(p, x - 1, y, XB.hy[t - L], e1_l, e1_c, phy_l, dummy);
    st4(hxw + at, hxb);
    st4(hyw + at, hyb);
    if (sx) st4(psi_hx_out + ((size_t)sp.hy_row(y) * nx + x) * L + lo, phx);
    if (sy2) st4(psi_hy_out + ((size_t)y * 2 * n + hxs) * L + lo, phy_c);
    float4 kq[NQ], jq[NQ], jm[NLQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      kq[q] = pv_kq[q];
      jq[q] = pv_jq[q];
    }
#pragma unroll
    for (int q = 0; q < NLQ; ++q) jm[q] = pv_jm[q];
    float4 pex = pv_pex, pey = pv_pey;
    uint32_t fl;
    float4 e2 = e_step<GEN, ND, NL>(p, x, y, e1_c, hyb - hybl, hxb - hxb_prev, pv_cf, kq, jq, jm, pex, pey, fl);
    if (NP > 0 && (fl & kF9)) {
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        const size_t ja = (q * plane + (size_t)y * nx + x) * L + lo;
        st4(J + ja, jq[q]);
        if (RR && q < ND && p.save_j) st4(save_j_slot(p, step + 2, g) + ja, jq[q]);
      }
#pragma unroll
      for (int q = 0; q < NL; ++q) st4(Jp + (q * plane + (size_t)y * nx + x) * L + lo, jm[q]);
    }
    if (fl & kEX) st4(psi_ezx + ((size_t)y * 2 * n + ex_s) * L + lo, pex);
    if (fl & kEY) st4(psi_ezy + ((size_t)sp.ey_row(y) * nx + x) * L + lo, pey);
    if (RR && (PK ? (src_rows >> (y - ya0)) & 1 : src_row)) add_sources(p, e2, x, y, lane_g, step + 1);
    if (RR && (PK ? (prb_rows >> (y - ya0)) & 1 : prb_row)) record_probes(p, e2, x, y, lane_g, step + 1);
    st4(ezw + at, e2);
    if (RR && p.save_ez) st4(save_ez_slot(p, step + 2, g) + at, e2);
    hxb_prev = hxb;
  };

  // The ring position of row slice k+1 and the slot of slice k, k counting
  // the slices from 0 (row rs).
  RingPos<NS> up{0, 0u};
  int cs = 0;
  wait(up);
  up.advance();
  const int k0 = ya0 > 0 ? 1 : 0;  // slices before A's first row
  if (ya0 > 0) {  // slot 0 holds row ya0-1: A's Hx^{n+1/2}(x, ya0-1)
    wait(up);
    if (valid && !aborted) {
      const Stage2d<L, NP, NL, PSI>& A = st[0];
      hxa_prev = hx_new<GEN>(p, GEN ? A.phx[cx * L + lo] : f4(0.f), nullptr, x, ya0 - 1, A.hx[cx * L + lo],
                             A.ez[(cx + 1) * L + lo], st[up.slot].ez[(cx + 1) * L + lo]);
    }
    release(cs);
    cs = up.slot;
    up.advance();
  }
  const int r_up = ya0 + nslots - 1 - k0;  // rows below r_up have the next slice in the ring

  // Source/probe bits of A's row r and of B's row r-1.  The single-grid
  // kernel shifts copies of the masks by one row per iteration; the packed
  // kernel (its parameters held in shared memory leave fewer registers) tests
  // bit r - ya0 of the masks in place.
  uint64_t srcm = src_rows, prbm = prb_rows;
  bool src_prev = false, prb_prev = false;

  for (int r = ya0; r < ya1; ++r) {
    const bool has_up = r < r_up;
    if (has_up) wait(up);
    float4 a_e = f4(0.f), a_hy = f4(0.f), a_phy = f4(0.f);
    float4 c_hx = f4(0.f), c_cf = f4(0.f), c_phx = f4(0.f), c_pex = f4(0.f), c_pey = f4(0.f);
    float4 kq[NQ], jq[NQ], jm[NLQ];
#pragma unroll
    for (int q = 0; q < NQ; ++q) kq[q] = jq[q] = f4(0.f);
#pragma unroll
    for (int q = 0; q < NLQ; ++q) jm[q] = f4(0.f);
    // Interior blocks compute step A unconditionally (every column is valid;
    // after an abort the values are never stored), so the zero defaults
    // above fold away on that path.
    if (!GEN || (valid && !aborted)) {
      // step A on row r: the one-step consumer's arithmetic
      const Stage2d<L, NP, NL, PSI>& A = st[cs];
      const int i0 = (cx + 1) * L + lo;
      const float4 ez_c = A.ez[i0];
      const float4 ez_up = has_up ? st[up.slot].ez[i0] : f4(0.f);
      bool sx, sy2, dummy;
      c_phx = GEN ? A.phx[cx * L + lo] : f4(0.f);  // psi slices: general path only
      const float4 hxn = hx_step<GEN>(p, x, r, A.hx[cx * L + lo], ez_c, ez_up, c_phx, sx);
      a_phy = GEN ? A.phy[i0] : f4(0.f);
      const float4 hyn = hy_step<GEN>(p, x, r, A.hy[i0], ez_c, A.ez[i0 + L], a_phy, sy2);
      float4 hyl = f4(0.f);
      if (!GEN || x >= 1) {
        float4 pl = GEN ? A.phy[i0 - L] : f4(0.f);
        hyl = hy_step<GEN>(p, x - 1, r, A.hy[i0 - L], A.ez[i0 - L], ez_c, pl, dummy);
      }
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        kq[q] = A.ade[q * CX + cx];
        jq[q] = A.j[(q * CX + cx) * L + lo];
      }
#pragma unroll
      for (int q = 0; q < NL; ++q) jm[q] = A.jp[(q * CX + cx) * L + lo];
      c_pex = GEN ? A.pex[cx * L + lo] : f4(0.f);
      c_pey = GEN ? A.pey[cx * L + lo] : f4(0.f);
      c_cf = A.coef[cx];
      uint32_t fl;
      a_e = e_step<GEN, ND, NL>(p, x, r, ez_c, hyn - hyl, hxn - hxa_prev, c_cf, kq, jq, jm, c_pex, c_pey, fl);
      if (RR && (PK ? (src_rows >> (r - ya0)) & 1 : srcm & 1)) add_sources(p, a_e, x, r, lane_g, step);
      if (own && !aborted && r >= y0 && r < y1) {
        if (RR && (PK ? (prb_rows >> (r - ya0)) & 1 : prbm & 1)) record_probes(p, a_e, x, r, lane_g, step);
        if (RR && p.save_ez) {  // the adjoint's copy of step n+1 (own cells)
          const size_t at = ((size_t)r * nx + x) * L + lo;
          st4(save_ez_slot(p, step + 1, g) + at, a_e);
          if (NP > 0 && p.save_j && (fl & kF9)) {
#pragma unroll
            for (int q = 0; q < ND; ++q) st4(save_j_slot(p, step + 1, g) + q * plane * L + at, jq[q]);
          }
        }
      }
      a_hy = hyn;
      c_hx = hxn;
      hxa_prev = hxn;
    }
    Exch2<L>& X = xr[r & 1];
    X.e[t] = a_e;
    X.hy[t] = a_hy;
    X.phy[t] = a_phy;
    // step B on row r-1 (or, for r-1 = y0-1, its Hx^{n+3/2} only); its
    // exchange row was written before the previous iteration's barrier
    const int y = r - 1;
    if (own && !aborted && y >= 0 && y >= y0 - 1 && y < y1) {
      if (y == y0 - 1) {
        float4 ps = pv_phx;
        bool dummy;
        hxb_prev = hx_step<GEN>(p, x, y, pv_hx, xr[y & 1].e[t], a_e, ps, dummy);
      } else {
        b_row(y, a_e, src_prev, prb_prev);
      }
    }
    if (!PK) {
      src_prev = srcm & 1;
      prb_prev = prbm & 1;
      srcm >>= 1;
      prbm >>= 1;
    }
    pv_hx = c_hx;
    pv_cf = c_cf;
    pv_phx = c_phx;
    pv_pex = c_pex;
    pv_pey = c_pey;
#pragma unroll
    for (int q = 0; q < NQ; ++q) {
      pv_kq[q] = kq[q];
      pv_jq[q] = jq[q];
    }
#pragma unroll
    for (int q = 0; q < NLQ; ++q) pv_jm[q] = jm[q];
    release(cs);
    cs = up.slot;
    up.advance();
    consumer_barrier();
    if (*abort_flag) aborted = true;
  }
  if (ya1 - ya0 + k0 < nslots) release(cs);  // the Ez-only slot of row ya1
  // the last own row when no A row lies above it (y1 == ny)
  if (own && !aborted && ya1 == y1 && y1 - 1 >= y0) b_row(y1 - 1, f4(0.f), src_prev, prb_prev);
}

// A two-step block with ring slots of one kind: PSI (a frame block: full
// slots, kStages2 of them, the general code) or not (an interior block:
// psi-less slots, NS of them, the interior code).
template <int L, int ND, int NL, bool PK, bool PSI, int NS>
CEEP_D void step2_run(const Fdtd2dParams& p, int step, int par, int x0, int y0, int y1, int ya0, int ya1,
                      int g, unsigned char* smem_raw) {
  using St = Stage2d<L, ND + NL, NL, PSI>;
  St* st = reinterpret_cast<St*>(smem_raw);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NS * sizeof(St));
  uint64_t* empty = full + NS;
  Exch2<L>* xr = reinterpret_cast<Exch2<L>*>(empty + NS);
  volatile int* abort_flag = reinterpret_cast<volatile int*>(xr + 2);
  const int rs = ya0 > 0 ? ya0 - 1 : 0;
  const int nslots = (ya1 - rs) + (ya1 < p.ny ? 1 : 0);

  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kConsumers / 32);
    }
    mbar_init_fence();
    *abort_flag = 0;
  }
  __syncthreads();
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");

  if (threadIdx.x >= kConsumers) {
    if (threadIdx.x == kConsumers) produce<L, ND, NL, NS, PSI>(p, st, full, empty, par, x0, ya0, ya1, rs, nslots, g);
    return;
  }
  if constexpr (PSI) {
    consume2<L, true, ND, NL, PK, true, true, NS>(p, st, full, empty, xr, abort_flag, step, par, x0, y0, y1, ya0,
                                                  ya1, rs, nslots, g);
  } else {
    // a block with no source/probe row and no adjoint save runs a loop
    // compiled without those paths (smaller code)
    bool rare = p.save_ez != nullptr;
    for (int y = ya0; !rare && y < ya1; ++y) rare = (__ldg(p.row_flags + y) & 3) != 0;
    if (!rare)
      consume2<L, false, ND, NL, PK, false, false, NS>(p, st, full, empty, xr, abort_flag, step, par, x0, y0, y1,
                                                       ya0, ya1, rs, nslots, g);
    else
      consume2<L, false, ND, NL, PK, false, true, NS>(p, st, full, empty, xr, abort_flag, step, par, x0, y0, y1,
                                                      ya0, ya1, rs, nslots, g);
  }
}

// One block of the two-step kernel: thread columns x0 .. x0+CX-1 (outputs
// x0+1 .. x0+CX-2), own rows y0 .. y0+rows2-1, TX group g.  Block-uniform:
// a block whose every cell, recomputed halo H included, lies in the plain
// interior of all regions (or any block of the interior-tile kernel, INT)
// runs the interior code on a deeper ring of psi-less slots; the far
// column/row is excluded too (Hy(nx-1), Hx(ny-1) are never updated and Ez
// there is an edge).
template <int L, int ND, int NL, bool PK, bool INT = false>
CEEP_D void step2_block(const Fdtd2dParams& p, int step, int par, int x0, int y0, int rows, int g,
                        unsigned char* smem_raw) {
  constexpr int CX = kConsumers / L;
  const int ny = p.ny, n = p.n;
  const int y1 = min(y0 + rows, ny);
  if (y0 >= y1) return;  // an empty piece of a short last tile row
  const int ya0 = y0 > 0 ? y0 - 1 : 0, ya1 = y1 < ny ? y1 + 1 : ny;  // step A's rows
  const int m = n > 1 ? n : 1;
  const bool interior = INT || ((x0 >= n + 1) && (x0 + CX <= p.nx - m) && (ya0 >= n + 1) && (ya1 <= ny - m));
  static_assert(step2_layout_bytes<L, ND, NL, false, interior_stages2<L, ND, NL>()>() <=
                    step2_layout_bytes<L, ND, NL, true, kStages2>(),
                "interior slots must fit the general blocks' shared memory");
  if (interior)
    step2_run<L, ND, NL, PK, false, interior_stages2<L, ND, NL>()>(p, step, par, x0, y0, y1, ya0, ya1, g, smem_raw);
  else if constexpr (!INT)
    step2_run<L, ND, NL, PK, true, kStages2>(p, step, par, x0, y0, y1, ya0, ya1, g, smem_raw);
}

template <int L, int ND, int NL>
__global__ void __launch_bounds__(kConsumers + 32, CEEP_MIN_BLOCKS2) fdtd2d_step2_kernel(const Fdtd2dParams p, int step, int par) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int CX = kConsumers / L;
  // frame tiles first, then the interior row-major: neighbouring interior
  // tiles, which share halo rows and columns, run close together in time
  // (their halos hit in L2)
  // Frame tiles run as p.fpieces2 blocks of about four rows each: a frame
  // tile takes several times an interior tile's time, and shorter, more
  // numerous frame blocks end sooner (the launch's last frame block sets its
  // length on small grids).
  const int fp = p.fpieces2;
  const int b = (int)blockIdx.x, nfp = fp * p.nframe2;
  const int tb = b < nfp ? b / fp : b - nfp + p.nframe2;
  int bx, by;
  tile_frame_first(tb, (p.nx + CX - 3) / (CX - 2), (p.ny + p.rows2 - 1) / p.rows2, p.frame2[0], p.frame2[1],
                   p.frame2[2], p.frame2[3], bx, by);
  int y0 = by * p.rows2, rows = p.rows2;
  if (b < nfp) {
    const int piece = b % fp;
    y0 += piece * p.rows2 / fp;
    rows = (piece + 1) * p.rows2 / fp - piece * p.rows2 / fp;
  }
  step2_block<L, ND, NL, false>(p, step, par, bx * (CX - 2) - 1, y0, rows, (int)blockIdx.z, smem_raw);
}

// The interior tiles of a split two-step launch (tiles nframe2 .. of the
// frame-first order; fdtd2d_step2_kernel runs tiles 0 .. nframe2-1 beside it
// on another stream).  Without the strip code and the psi slices a block
// needs fewer registers and less shared memory, so four blocks share an SM
// (three with two ADE poles) against three of the general kernel.  Not the
// default: while the long frame blocks run, an SM holding one of them has
// room for only two interior blocks, and the two kernels' step boundary is a
// full join without programmatic dependent launch; on the 600^2 x 16 head
// the split launch measured 31.5 us per step against 29.7 for one kernel.
template <int L, int ND, int NL>
__global__ void __launch_bounds__(kConsumers + 32, ND + NL >= 2 ? CEEP_MIN_BLOCKS2 : CEEP_MIN_BLOCKS2I)
    fdtd2d_step2i_kernel(const Fdtd2dParams p, int step, int par) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  constexpr int CX = kConsumers / L;
  int bx, by;
  tile_frame_first(p.nframe2 + (int)blockIdx.x, (p.nx + CX - 3) / (CX - 2), (p.ny + p.rows2 - 1) / p.rows2,
                   p.frame2[0], p.frame2[1], p.frame2[2], p.frame2[3], bx, by);
  step2_block<L, ND, NL, false, true>(p, step, par, bx * (CX - 2) - 1, by * p.rows2, p.rows2, (int)blockIdx.z,
                                      smem_raw);
}

// Many phantoms, two steps per launch: block b runs two-step tile
// tiles_a[b] for b < na, else tiles_b[b - na] (the frame tiles of every
// running phantom first, then their interior tiles; x0 = the tile's first
// thread column) of phantom t.phantom.
template <int L, int ND, int NL>
__global__ void __launch_bounds__(kConsumers + 32, CEEP_MIN_BLOCKS2)
    fdtd2d_packed2_kernel(const PackTile* __restrict__ tiles_a, int na, const PackTile* __restrict__ tiles_b,
                          const Fdtd2dParams* __restrict__ params, int step, int par) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(16) Fdtd2dParams sp;
  const int b = (int)blockIdx.x;
  const PackTile t = b < na ? tiles_a[b] : tiles_b[b - na];
  const int* src = reinterpret_cast<const int*>(params + t.phantom);
  int* dst = reinterpret_cast<int*>(&sp);
  for (int i = threadIdx.x; i < (int)(sizeof(Fdtd2dParams) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  step2_block<L, ND, NL, true>(sp, step, par, t.x0, t.y0, t.rows, t.g, smem_raw);
}

// Many phantoms in one launch: block b runs tile tiles[b] of phantom
// tiles[b].phantom, whose parameters are staged into shared memory first
// (they are constant, so this happens before the dependency wait).
template <int L, int ND, int NL>
__global__ void __launch_bounds__(kConsumers + 32, CEEP_MIN_BLOCKS)
    fdtd2d_packed_kernel(const PackTile* __restrict__ tiles_a, int na, const PackTile* __restrict__ tiles_b,
                         const Fdtd2dParams* __restrict__ params, int step, int par) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  __shared__ __align__(16) Fdtd2dParams sp;
  const int b = (int)blockIdx.x;
  const PackTile t = b < na ? tiles_a[b] : tiles_b[b - na];
  const int* src = reinterpret_cast<const int*>(params + t.phantom);
  int* dst = reinterpret_cast<int*>(&sp);
  for (int i = threadIdx.x; i < (int)(sizeof(Fdtd2dParams) / sizeof(int)); i += blockDim.x) dst[i] = src[i];
  __syncthreads();
  step_block<L, ND, NL>(sp, step, par, t.x0, t.y0, t.g, smem_raw);
}

// ------------------------------------------------------------------------
// Host side: launch configuration and the rows-per-block choice.
// ------------------------------------------------------------------------
// Frame tile counts (left, right, top, bottom) of a tile grid whose column
// bx starts at cell x0(bx) with `cw` thread columns and whose row by covers
// `rows` cells (`halo`: the two-step kernel's step A rows reach one row
// beyond each side), using the kernels' own interior tests.
static void frame_counts(const Fdtd2dParams& p, int cw, int xstep, int xoff, int rows, bool halo, int out[4]) {
  const int n = p.n, m = n > 1 ? n : 1;
  const int gx = (p.nx + (halo ? cw - 3 : cw - 1)) / xstep, gy = (p.ny + rows - 1) / rows;
  auto in_x = [&](int bx) { const int x0 = bx * xstep + xoff; return x0 >= n + 1 && x0 + cw <= p.nx - m; };
  auto in_y = [&](int by) {
    const int y0 = by * rows, y1 = y0 + rows < p.ny ? y0 + rows : p.ny;
    const int a0 = halo ? (y0 > 0 ? y0 - 1 : 0) : y0, a1 = halo ? (y1 < p.ny ? y1 + 1 : p.ny) : y1;
    return a0 >= n + 1 && a1 <= p.ny - m;
  };
  int fl = 0, fr = 0, ft = 0, fb = 0;
  while (fl < gx && !in_x(fl)) ++fl;
  while (fr < gx - fl && !in_x(gx - 1 - fr)) ++fr;
  while (ft < gy && !in_y(ft)) ++ft;
  while (fb < gy - ft && !in_y(gy - 1 - fb)) ++fb;
  out[0] = fl; out[1] = fr; out[2] = ft; out[3] = fb;
}

template <int L, int ND, int NL>
static cudaError_t configure_l(Fdtd2dParams& p) {
  constexpr size_t smem = stage_smem_bytes<L, ND + NL, NL>();
  auto kern = fdtd2d_step_kernel<L, ND, NL>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  p.smem = (int)smem;
  if (p.rows > kMaxRows) p.rows = kMaxRows;
  if (p.rows <= 0) {
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kConsumers + 32, smem);
    if (e != cudaSuccess) return e;
    p.rows = choose_rows(p.nx, p.ny, p.groups, kConsumers / L, (long)sms * (per_sm < 1 ? 1 : per_sm), kMaxRows);
  }
  frame_counts(p, kConsumers / L, kConsumers / L, 0, p.rows, false, p.frame1);
  return cudaSuccess;
}

// The two-step kernel: shared memory, and rows per block (its A rows add two
// halo rows to the segment, which stays <= 62 so the row masks hold 64).
template <int L, int ND, int NL>
static cudaError_t configure2_l(Fdtd2dParams& p) {
  constexpr size_t smem = step2_smem_bytes<L, ND, NL>();
  auto kern = fdtd2d_step2_kernel<L, ND, NL>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  p.smem2 = (int)smem;
  int dev = 0, sms = 148, per_sm = 1;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kConsumers + 32, smem);
  if (e != cudaSuccess) return e;
  // a tile height given by the caller applies to both kernels
  p.rows2 = p.rows_fixed > 0 ? (p.rows_fixed < 62 ? p.rows_fixed : 62)
                             : choose_rows(p.nx, p.ny, p.groups, kConsumers / L - 2,
                                           (long)sms * (per_sm < 1 ? 1 : per_sm), 62);
  frame_counts(p, kConsumers / L, kConsumers / L - 2, -1, p.rows2, true, p.frame2);
  // the interior-tile kernel of a split launch, and the frame tile count
  constexpr size_t smem_i = step2_smem_bytes<L, ND, NL, false>();
  e = cudaFuncSetAttribute(fdtd2d_step2i_kernel<L, ND, NL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem_i);
  if (e != cudaSuccess) return e;
  p.smem2i = (int)smem_i;
  constexpr int CX = kConsumers / L;
  const int gx = (p.nx + CX - 3) / (CX - 2), gy = (p.ny + p.rows2 - 1) / p.rows2;
  const int ic = gx - p.frame2[0] - p.frame2[1], ir = gy - p.frame2[2] - p.frame2[3];
  p.ntiles2 = gx * gy;
  // frame tiles as pieces of about four rows (measured at 600^2 x 16:
  // 10-row tiles in 2 pieces, 12-row tiles in 3)
  p.fpieces2 = p.rows2 >= 8 ? p.rows2 / 4 : 1;
  p.nframe2 = gx * gy - (ic > 0 && ir > 0 ? ic * ir : 0);
  return cudaSuccess;
}

// Two steps.  Split (a side stream given, p.split2 set, both kinds of tile
// present): the frame tiles run as fdtd2d_step2_kernel on the side stream
// (forked from and joined back to s) beside the interior tiles as
// fdtd2d_step2i_kernel on s; both read the state of [par] and write disjoint
// tiles of [par^1].  Otherwise one launch of every tile, with programmatic
// dependent launch on the previous step.
template <int L, int ND, int NL>
static cudaError_t launch2_l(const Fdtd2dParams& p, int step, int par, cudaStream_t s, const Fdtd2dSide* side) {
  const int ntiles = p.ntiles2, ninterior = ntiles - p.nframe2;
  if (side && p.split2 && p.nframe2 > 0 && ninterior > 0) {
    cudaError_t e;
    if ((e = cudaEventRecord(side->fork, s)) != cudaSuccess) return e;
    if ((e = cudaStreamWaitEvent(side->stream, side->fork, 0)) != cudaSuccess) return e;
    cudaLaunchConfig_t cf = {};
    cf.gridDim = dim3(p.fpieces2 * p.nframe2, 1, p.groups);
    cf.blockDim = dim3(kConsumers + 32);
    cf.dynamicSmemBytes = p.smem2;
    cf.stream = side->stream;
    if ((e = cudaLaunchKernelEx(&cf, fdtd2d_step2_kernel<L, ND, NL>, p, step, par)) != cudaSuccess) return e;
    cudaLaunchConfig_t ci = cf;
    ci.gridDim = dim3(ninterior, 1, p.groups);
    ci.dynamicSmemBytes = p.smem2i;
    ci.stream = s;
    if ((e = cudaLaunchKernelEx(&ci, fdtd2d_step2i_kernel<L, ND, NL>, p, step, par)) != cudaSuccess) return e;
    if ((e = cudaEventRecord(side->join, side->stream)) != cudaSuccess) return e;
    return cudaStreamWaitEvent(s, side->join, 0);
  }
  dim3 grid(ntiles + (p.fpieces2 - 1) * p.nframe2, 1, p.groups);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(kConsumers + 32);
  cfg.dynamicSmemBytes = p.smem2;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, fdtd2d_step2_kernel<L, ND, NL>, p, step, par);
}

template <int L, int ND, int NL>
static cudaError_t launch_l(const Fdtd2dParams& p, int step, int par, cudaStream_t s) {
  constexpr int CX = kConsumers / L;
  dim3 grid(((p.nx + CX - 1) / CX) * ((p.ny + p.rows - 1) / p.rows), 1, p.groups);
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = dim3(kConsumers + 32);
  cfg.dynamicSmemBytes = p.smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, fdtd2d_step_kernel<L, ND, NL>, p, step, par);
}

template <int L, int ND, int NL>
static cudaError_t launch_packed_l(const PackTile* tiles_a, int na, const PackTile* tiles_b, int nb,
                                   const Fdtd2dParams* params, int step, int par, bool two, cudaStream_t s) {
  const size_t smem = two ? step2_smem_bytes<L, ND, NL>() : stage_smem_bytes<L, ND + NL, NL>();
  static bool attr_set[2] = {false, false};
  if (!attr_set[two]) {
    cudaError_t e = two ? cudaFuncSetAttribute(fdtd2d_packed2_kernel<L, ND, NL>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem)
                        : cudaFuncSetAttribute(fdtd2d_packed_kernel<L, ND, NL>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_set[two] = true;
  }
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(na + nb);
  cfg.blockDim = dim3(kConsumers + 32);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (two) return cudaLaunchKernelEx(&cfg, fdtd2d_packed2_kernel<L, ND, NL>, tiles_a, na, tiles_b, params, step, par);
  return cudaLaunchKernelEx(&cfg, fdtd2d_packed_kernel<L, ND, NL>, tiles_a, na, tiles_b, params, step, par);
}

template <int ND, int NL>
cudaError_t fdtd2d_packed_poles(int L, const PackTile* ta, int na, const PackTile* tb, int nb,
                                const Fdtd2dParams* params, int step, int par, bool two, cudaStream_t s) {
  switch (L) {
    case 1: return launch_packed_l<1, ND, NL>(ta, na, tb, nb, params, step, par, two, s);
    case 2: return launch_packed_l<2, ND, NL>(ta, na, tb, nb, params, step, par, two, s);
    case 4: return launch_packed_l<4, ND, NL>(ta, na, tb, nb, params, step, par, two, s);
    default: return launch_packed_l<8, ND, NL>(ta, na, tb, nb, params, step, par, two, s);
  }
}

// what: 0 = configure, 1 = one step, 2 = two steps
template <int L, int ND, int NL>
static cudaError_t act_l(Fdtd2dParams& p, int step, int par, cudaStream_t s, int what, const Fdtd2dSide* side) {
  if (what == 0) {
    cudaError_t e = configure_l<L, ND, NL>(p);
    return e != cudaSuccess ? e : configure2_l<L, ND, NL>(p);
  }
  return what == 1 ? launch_l<L, ND, NL>(p, step, par, s) : launch2_l<L, ND, NL>(p, step, par, s, side);
}

template <int ND, int NL>
cudaError_t fdtd2d_dispatch_poles(Fdtd2dParams& p, int step, int par, cudaStream_t s, int what,
                                  const Fdtd2dSide* side) {
  switch (p.L) {
    case 1: return act_l<1, ND, NL>(p, step, par, s, what, side);
    case 2: return act_l<2, ND, NL>(p, step, par, s, what, side);
    case 4: return act_l<4, ND, NL>(p, step, par, s, what, side);
    default: return act_l<8, ND, NL>(p, step, par, s, what, side);
  }
}

}  // namespace ceep

// Explicit instantiation of one ADE shape's launch and configure entry points
// (and through them every kernel of that shape).
#define CEEP_FDTD2D_INSTANTIATE(ND, NL)                                                                        \
  namespace ceep {                                                                                           \
  template cudaError_t fdtd2d_dispatch_poles<ND, NL>(Fdtd2dParams&, int, int, cudaStream_t, int,             \
                                                     const Fdtd2dSide*);                                     \
  template cudaError_t fdtd2d_packed_poles<ND, NL>(int, const PackTile*, int, const PackTile*, int,           \
                                                   const Fdtd2dParams*, int, int, bool, cudaStream_t);        \
  }

// Exact discrete adjoint of the fused 2D step (sm_100a): one launch per step.
//
// The forward step (fdtd2d_kernels.cuh, after fdtd_2d_batched.py:454-526) is a chain
// of linear maps; the transposed step applies their transposes in reverse
// order.  Per cell it has two halves:
//
//   E half (pointwise): probe-gradient injection, edge zeroing, transposed
//     E-CPML psi recurrences, transposed interior E update and Debye current
//     recurrence.  It yields the adjoints of the two curls at the cell (cy of
//     Hy(x)-Hy(x-1), cx of Hx(y)-Hx(y-1)) and the pointwise part of the E
//     adjoint, and adds this step's per-cell parameter gradients:
//       dE1/dca = E^n, dE1/dcb = (E1 - ca E^n)/cb, dJ'/dk1 = J^n,
//       dJ'/dk2 = (E1 - E^n)/dt, dE1/dgamma = -cb J^n,
//     where E1 is the interior update (E^{n+1} minus the source).
//   H half (5-point): transposed curls and H updates with the strip psi
//     recurrences, and the gather of the E adjoint from the H differences
//     E(x+1)-E(x), E(y+1)-E(y) of the cell and of its left and lower
//     neighbours.
//
// Schedule (the forward kernel's): a block owns a column strip of CX cells
// and a segment of rows; one producer thread streams each row's slices into a
// shared-memory ring with 1D bulk copies (cp.async.bulk, no multicast); 128
// consumer threads walk the rows upward.  At row y a thread runs the E half
// of row y+1 and the H half of row y, so the curl adjoints never leave the
// chip: cx(y) and the lower neighbour's contribution to the E adjoint are
// carried in registers, cy of the left and right neighbours comes from the
// neighbouring lanes by shuffle, and the lanes at a warp edge recompute the
// one neighbour cy they miss from the staged row (which carries a one-cell
// halo).  The rows just below and above the segment are recomputed (E half,
// cx only), never exchanged; every adjoint array is ping-pong buffered so
// those recomputes read values no other block is writing.
//
// Gradients are exact for the interior E region (where the update
// coefficients act); the E-CPML scale dt/(eps_r eps0) of strip cells is not
// differentiated (the ADE and phantom live in the interior by construction).
// Every mbarrier wait is bounded in time; on expiry the block records
// CEEP_ERR_TIMEOUT in the status word and returns.
#include "../../include/ceep_b200.h"
#include "adjoint2d.cuh"
#include "common.cuh"
#include "tma.cuh"

namespace ceep {

constexpr int kAdjConsumers = 128;
// Resident blocks per SM the registers are budgeted for, and the ring depth
// (stages are shrunk from 4 to 3 when 4 would not fit that many blocks).
#ifndef CEEP_ADJ_MIN_BLOCKS
#define CEEP_ADJ_MIN_BLOCKS 3
#endif
constexpr int kAdjMaxRows = 62;                  // rows + the two neighbour rows fit a 64-bit row mask
constexpr uint64_t kAdjWaitNs = 1000000000ull;   // 1 s

template <int L>
CEEP_D float lane_sum(float v) {
#pragma unroll
  for (int o = L / 2; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
CEEP_D float dot4(float4 a, float4 b) { return a.x * b.x + a.y * b.y + a.z * b.z + a.w * b.w; }
CEEP_D float4 shfl_up4(float4 v, int d) {
  return make_float4(__shfl_up_sync(0xffffffffu, v.x, d), __shfl_up_sync(0xffffffffu, v.y, d),
                     __shfl_up_sync(0xffffffffu, v.z, d), __shfl_up_sync(0xffffffffu, v.w, d));
}
CEEP_D float4 shfl_down4(float4 v, int d) {
  return make_float4(__shfl_down_sync(0xffffffffu, v.x, d), __shfl_down_sync(0xffffffffu, v.y, d),
                     __shfl_down_sync(0xffffffffu, v.z, d), __shfl_down_sync(0xffffffffu, v.w, d));
}

// One slot of the ring: the slices of one row.  Halo'd slices hold cells
// x0-1 .. x0+CX, left-halo'd ones x0-1 .. x0+CX-1, the rest x0 .. x0+CX-1.
// The CPML psi slices are not staged: only strip cells read them, straight
// from the read half of their ping-pong pair, which keeps a stage small
// enough for three blocks per SM.
template <int L, int ND, int NL>
struct AdjStage {
  static constexpr int CX = kAdjConsumers / L;
  static constexpr int H = CX + 2;
  static constexpr int NP = ND + NL;  // poles: the Debye ones first, then the Lorentz ones
  static constexpr int NQ = NP > 0 ? NP : 1;
  float4 le[H * L];                        // adjoint Ez (halo'd)
  float4 lj[NQ * H * L];                   // adjoint currents of every pole (halo'd)
  float4 coef[H];                          // ca, cb, dt/(eps_r eps0), 0 (halo'd)
  float4 ade[NQ * H];                      // Debye (k1, k2, gamma, 0), Lorentz (k1, k2, k3, 0) (halo'd)
  float4 en[CX * L];                       // forward Ez^n
  float4 e1[CX * L];                       // forward Ez^{n+1}
  float4 jn[ND > 0 ? ND * CX * L : 1];     // forward Debye J^n (tau gradients)
  float4 ljp[NL > 0 ? NL * CX * L : 1];    // adjoint Lorentz J_prev
  float4 lhx[CX * L];                      // adjoint Hx
  float4 lhy[(CX + 1) * L];                // adjoint Hy (left-halo'd)
};

// Four stages where CEEP_ADJ_MIN_BLOCKS blocks of them fit an SM, else three.
template <int L, int ND, int NL>
__host__ __device__ constexpr int adj_stages() {
  return 4 * sizeof(AdjStage<L, ND, NL>) <= (222 / CEEP_ADJ_MIN_BLOCKS) * 1024 ? 4 : 3;
}
template <int L, int ND, int NL>
__host__ __device__ constexpr size_t adj_smem_bytes() {
  return adj_stages<L, ND, NL>() * sizeof(AdjStage<L, ND, NL>) + 2 * adj_stages<L, ND, NL>() * sizeof(uint64_t);
}

CEEP_D void adj_status(int* status, int code) {
  if (status) atomicCAS(status, 0, code);
}

// Region predicates of the forward step (fdtd2d_kernels.cuh) for one cell.
struct AdjRegions {
  int n, nx, ny;
  CEEP_D bool f9(int x, int y) const { return x >= n + 1 && x < nx - n && y >= n + 1 && y < ny - n; }
  CEEP_D bool edge(int x, int y) const { return x == 0 || x == nx - 1 || y == 0 || y == ny - 1; }
  // E-CPML y strips (rows 1..n, ny-n..ny-1): strip row or -1, profile index
  CEEP_D int ey_row(int y) const {
    return (y >= 1 && y <= n) ? y - 1 : (n > 0 && y >= ny - n) ? n + (y - (ny - n)) : -1;
  }
  CEEP_D int ey_ci(int y) const { return y <= n ? y - 1 : ny - 1 - y; }
  // E-CPML x strips (columns 1..n, nx-n..nx-1)
  CEEP_D int ex_col(int x) const {
    return (x >= 1 && x <= n) ? x - 1 : (n > 0 && x >= nx - n) ? n + (x - (nx - n)) : -1;
  }
  CEEP_D int ex_ci(int x) const { return x <= n ? x - 1 : nx - 1 - x; }
  // H-CPML y strips of Hx (rows y < n, ny-n <= y < ny-1)
  CEEP_D int hy_row(int y) const { return y < n ? y : (y >= ny - n && y < ny - 1) ? n + (y - (ny - n)) : -1; }
  // H-CPML x strips of Hy (columns x < n, nx-n <= x < nx-1)
  CEEP_D int hx_col(int x) const { return x < n ? x : (x >= nx - n && x < nx - 1) ? n + (x - (nx - n)) : -1; }
};

// Transposed H update of one cell.  tot = adjoint of H' in total, u = adjoint
// of the forward difference the update reads, psi = adjoint of the old psi
// (strip cells, s >= 0 = strip index).
struct HAdj {
  float4 tot, psi, u;
  int s;
};

// Hy' = Hy + A (E(x+1) - E(x)) [+ db psi'],  psi' = b psi + c/dx (E(x+1) - E(x))
// `psi` is the adjoint psi of the cell (read by the caller ahead of the row's
// stores; used by strip cells only).
template <bool GEN>
CEEP_D HAdj hy_adj(const Fdtd2dParams& p, const AdjRegions& rg, int x, int y, float4 lhy, float4 cy_c, float4 cy_r,
                   float4 psi) {
  HAdj r;
  r.tot = lhy + cy_c - cy_r;
  r.s = -1;
  if (!GEN) {
    r.u = p.db_dx * r.tot;
    return r;
  }
  const float A = (x >= p.n && x < p.nx - 1 && y >= p.n && y < p.ny - p.n) ? p.db_dx : 0.f;
  r.u = A * r.tot;
  r.s = rg.hx_col(x);
  if (r.s >= 0) {
    const int ci = x < p.n ? x : p.nx - 1 - x;
    const float4 pt = fma4(p.db, r.tot, psi);
    r.psi = p.cpml_b[ci] * pt;
    r.u = fma4(p.cpml_c[ci] * p.inv_dx, pt, r.u);
  }
  return r;
}

// Hx' = Hx - A (E(y+1) - E(y)) [- db psi'],  psi' = b psi + c/dx (E(y+1) - E(y))
template <bool GEN>
CEEP_D HAdj hx_adj(const Fdtd2dParams& p, const AdjRegions& rg, int x, int y, float4 lhx, float4 cx_c, float4 cx_u,
                   float4 psi) {
  HAdj r;
  r.tot = lhx + cx_c - cx_u;
  r.s = -1;
  if (!GEN) {
    r.u = (-p.db_dx) * r.tot;
    return r;
  }
  const float A = (x >= p.n && x < p.nx - p.n && y >= p.n && y < p.ny - 1) ? p.db_dx : 0.f;
  r.u = (-A) * r.tot;
  r.s = rg.hy_row(y);
  if (r.s >= 0) {
    const int ci = y < p.n ? y : p.ny - 1 - y;
    const float4 pt = fma4(-p.db, r.tot, psi);
    r.psi = p.cpml_b[ci] * pt;
    r.u = fma4(p.cpml_c[ci] * p.inv_dx, pt, r.u);
  }
  return r;
}

// p_n = Ez after step n at the probe cells: its adjoint enters here.
CEEP_D void inject_probes(const Adjoint2dParams& a, float4& E, int x, int y, int lane_g, int step) {
  const Fdtd2dParams& p = a.f;
  for (int q = 0; q < p.nprobe; ++q)
    if (__ldg(p.prb_xy + 2 * q) == x && __ldg(p.prb_xy + 2 * q + 1) == y) {
#pragma unroll
      for (int c = 0; c < 4; ++c) {
        const int tx = 4 * lane_g + c;
        if (tx < p.ntx) add_comp(E, c, __ldg(a.probe_grad + ((size_t)tx * p.nprobe + q) * p.nsteps + step));
      }
    }
}

// ------------------------------------------------------------------------
// Producer: one thread, bulk copies of row slices into the stage ring.
// Every row: adjoint Ez and J, coefficients (halo'd).  Rows of the segment
// and the one below it: adjoint Hx.  Rows of the segment: forward Ez^n,
// Ez^{n+1}, J^n and adjoint Hy.
// ------------------------------------------------------------------------
template <int L, int ND, int NL>
CEEP_D void adj_produce(const Adjoint2dParams& a, AdjStage<L, ND, NL>* st, uint64_t* full, uint64_t* empty, int par,
                        const float4* ez_n, const float4* ez_np1, const float4* j_n, int x0, int y0, int y1, int rs,
                        int nslots, int g) {
  using St = AdjStage<L, ND, NL>;
  constexpr int CX = St::CX, H = St::H, NS = adj_stages<L, ND, NL>();
  const Fdtd2dParams& p = a.f;
  const int nx = p.nx;
  const size_t gf = (size_t)g * p.gs_field, gj = (size_t)g * p.gs_j, gjp = (size_t)g * p.gs_jp;
  const size_t plane = (size_t)nx * p.ny;
  const float4* coef = reinterpret_cast<const float4*>(p.coef);
  const float4* ade = reinterpret_cast<const float4*>(p.ade_coef);
  constexpr int NP = ND + NL;
  const int xa = x0 > 0 ? x0 - 1 : 0;                  // first halo'd cell
  const int xb = x0 + CX + 1 < nx ? x0 + CX + 1 : nx;  // end of the halo'd cells
  const int xe = x0 + CX < nx ? x0 + CX : nx;          // end of the owned cells
  const int ha = xa - (x0 - 1);                         // slot index of cell xa
  const uint32_t cb = L * 16;
  int issued = 0;
  for (int k = 0; k < nslots; ++k) {
    const int s = k % NS, u = k / NS;
    if (u > 0 && !mbar_wait_bounded(&empty[s], (u - 1) & 1, kAdjWaitNs)) {
      adj_status(p.status, CEEP_ERR_TIMEOUT);
      break;
    }
    const int r = rs + k;
    const bool tail = r >= y1, body = r >= y0 && !tail;
    St& S = st[s];
    const size_t rowc = (size_t)r * nx;
    for (int pass = 0; pass < 2; ++pass) {
      uint32_t bytes = 0;
      auto cp = [&](void* dst, const void* src, uint32_t nb) {
        if (nb == 0) return;
        if (pass) bulk_g2s(dst, src, nb, &full[s]);
        else bytes += nb;
      };
      cp(S.le + ha * L, a.ez[par] + gf + (rowc + xa) * L, (xb - xa) * cb);
      cp(S.coef + ha, coef + rowc + xa, (xb - xa) * 16u);
#pragma unroll
      for (int q = 0; q < NP; ++q) {
        cp(S.ade + q * H + ha, ade + q * plane + rowc + xa, (xb - xa) * 16u);
        cp(S.lj + (q * H + ha) * L, a.j[par] + gj + (q * plane + rowc + xa) * L, (xb - xa) * cb);
      }
      if (!tail) cp(S.lhx, a.hx[par] + gf + (rowc + x0) * L, (xe - x0) * cb);
      if (body) {
        cp(S.en, ez_n + gf + (rowc + x0) * L, (xe - x0) * cb);
        cp(S.e1, ez_np1 + gf + (rowc + x0) * L, (xe - x0) * cb);
        if (a.grad_tau) {
#pragma unroll
          for (int q = 0; q < ND; ++q) cp(S.jn + q * CX * L, j_n + gj + (q * plane + rowc + x0) * L, (xe - x0) * cb);
        }
        cp(S.lhy + ha * L, a.hy[par] + gf + (rowc + xa) * L, (xe - xa) * cb);
#pragma unroll
        for (int q = 0; q < NL; ++q)
          cp(S.ljp + q * CX * L, a.jp[par] + gjp + (q * plane + rowc + x0) * L, (xe - x0) * cb);
      }
      if (!pass) mbar_arrive_expect_tx(&full[s], bytes);
    }
    issued = k + 1;
  }
  // Let every copy this thread issued land before it leaves.
  for (int k = issued > NS ? issued - NS : 0; k < issued; ++k)
    mbar_wait_bounded(&full[k % NS], (k / NS) & 1, kAdjWaitNs);
}

// E-half results of one cell carried between rows.
struct AdjE {
  float4 cx, cy;  // adjoints of the two curls at the cell
  float4 cye;     // warp-edge lanes: cy of the neighbour across the warp edge
  float4 elin;    // pointwise part of the E adjoint
};

// ------------------------------------------------------------------------
// Consumer: one float4 (4 TX) of one cell per thread, walking the rows.
// GEN = false for blocks whose cells, halo cells and neighbour rows all lie
// in the plain interior of every region.
// ------------------------------------------------------------------------
template <int L, int ND, int NL, bool GEN>
CEEP_D void adj_consume(const Adjoint2dParams& a, AdjStage<L, ND, NL>* st, uint64_t* full, uint64_t* empty, int step,
                        int par, int x0, int y0, int y1, int rs, int nslots, int g) {
  using St = AdjStage<L, ND, NL>;
  constexpr int CX = St::CX, H = St::H, NS = adj_stages<L, ND, NL>();
  constexpr int KG = 2 + 3 * (ND + NL), KP = adjoint2d_grad_width(ND + NL);
  const Fdtd2dParams& p = a.f;
  const int nx = p.nx, ny = p.ny, n = p.n;
  const AdjRegions rg{n, nx, ny};
  const int cx = threadIdx.x / L, lo = threadIdx.x % L;
  const int x = x0 + cx;
  const bool active = x < nx;
  const int lw = threadIdx.x & 31;
  const int lane_g = g * L + lo;
  const float inv = p.inv_dx;
  const size_t plane = (size_t)nx * ny, gf = (size_t)g * p.gs_field;
  const int me = cx * L + lo;        // this cell in the plain slices
  const int mh = (cx + 1) * L + lo;  // this cell in the halo'd slices
  // read and write halves of the psi pairs, at this TX group
  const float4* pex_r = a.psi_ezx[par] + (size_t)g * p.gs_psi_x;
  const float4* pey_r = a.psi_ezy[par] + (size_t)g * p.gs_psi_y;
  const float4* phy_r = a.psi_hy[par] + (size_t)g * p.gs_psi_x;
  const float4* phx_r = a.psi_hx[par] + (size_t)g * p.gs_psi_y;

  // Probe cells of this column and of the neighbour column an edge lane
  // recomputes, and this lane's source cells, among rows rs .. rs + nslots - 1
  // (<= 64) as bit masks; found once, before the first wait.
  const int xn = lw < L ? x - 1 : (lw >= 32 - L ? x + 1 : x);
  uint64_t prb_own = 0, prb_nb = 0, src_own = 0;
  for (int q = 0; q < p.nprobe; ++q) {
    const int px = __ldg(p.prb_xy + 2 * q), py = __ldg(p.prb_xy + 2 * q + 1) - rs;
    if (py >= 0 && py < nslots) {
      if (px == x) prb_own |= 1ull << py;
      if (px == xn) prb_nb |= 1ull << py;
    }
  }
  for (int s = 4 * lane_g; s < 4 * lane_g + 4 && s < p.ntx; ++s) {
    const int sx = __ldg(p.src_xy + 2 * s), sy = __ldg(p.src_xy + 2 * s + 1) - rs;
    if (sx == x && sy >= 0 && sy < nslots) src_own |= 1ull << sy;
  }

  auto wait = [&](int k) {
    const bool ok = mbar_wait_bounded(&full[k % NS], (k / NS) & 1, kAdjWaitNs);
    if (__any_sync(0xffffffffu, !ok)) {
      if (lw == 0) adj_status(p.status, CEEP_ERR_TIMEOUT);
      return false;
    }
    return true;
  };
  auto release = [&](int k) {
    __syncwarp();
    if (lw == 0) mbar_arrive(&empty[k % NS]);
  };
  // adjoint Ez of halo'd cell i (cell xc) of row r after probe injection and edge zeroing
  auto e_adj = [&](const St& S, int i, int xc, int r) {
    float4 E = S.le[i * L + lo];
    if (((xc == x ? prb_own : prb_nb) >> (r - rs)) & 1) inject_probes(a, E, xc, r, lane_g, step);
    if (GEN && rg.edge(xc, r)) E = f4(0.f);
    return E;
  };
  // sum over poles of (k2/dt) * adjoint J at halo'd cell i
  auto jsum = [&](const St& S, int i) {
    float4 s = f4(0.f);
#pragma unroll
    for (int q = 0; q < ND + NL; ++q) s = fma4(S.ade[q * H + i].y * p.inv_dt, S.lj[(q * H + i) * L + lo], s);
    return s;
  };
  // Adjoint psi of strip cells, read from the read halves of their pairs.  A
  // row's values are all loaded at the top of its iteration, ahead of any
  // store, so their latencies overlap each other and the shared-memory reads.
  auto ld_pey = [&](int xc, int r) {  // E y strips (rows 1..n, ny-n..ny-1; x >= 1)
    const int sy = rg.ey_row(r);
    return (GEN && n > 0 && xc >= 1 && xc < nx && sy >= 0) ? __ldg(pey_r + ((size_t)sy * nx + xc) * L + lo) : f4(0.f);
  };
  auto ld_pex = [&](int xc, int r) {  // E x strips (columns 1..n, nx-n..nx-1; y >= 1)
    const int sx = (xc >= 0 && xc < nx) ? rg.ex_col(xc) : -1;
    return (GEN && n > 0 && r >= 1 && sx >= 0) ? __ldg(pex_r + ((size_t)r * 2 * n + sx) * L + lo) : f4(0.f);
  };
  auto ld_phy = [&](int xc, int y) {  // H x strips of Hy
    const int sh = (xc >= 0 && xc < nx) ? rg.hx_col(xc) : -1;
    return (GEN && sh >= 0) ? __ldg(phy_r + ((size_t)y * 2 * n + sh) * L + lo) : f4(0.f);
  };
  auto ld_phx = [&](int y) {  // H y strips of Hx, this column
    const int sh = rg.hy_row(y);
    return (GEN && active && sh >= 0) ? __ldg(phx_r + ((size_t)sh * nx + x) * L + lo) : f4(0.f);
  };
  // the column an edge lane recomputes cy for (its own otherwise)
  const int x_nb = lw < L ? x - 1 : (lw >= 32 - L ? x + 1 : x);
  // cy of halo'd cell i (cell xc) of row r; pex = that cell's adjoint E x-strip psi
  auto cy_at = [&](const St& S, int i, int xc, int r, float4 pex) {
    const float4 E = e_adj(S, i, xc, r);
    const float4 cf = S.coef[i];
    if (!GEN || rg.f9(xc, r)) return (cf.y * inv) * (E + jsum(S, i));
    if (n > 0 && r >= 1) {
      const int sx = rg.ex_col(xc);
      if (sx >= 0) return (p.cpml_c[rg.ex_ci(xc)] * inv) * fma4(cf.z, E, pex);
    }
    return f4(0.f);
  };
  // cx of this cell in a neighbour row (r = y0 - 1 or y1); pey = its E y-strip psi
  auto cx_row = [&](const St& S, int r, float4 pey) {
    if (!active) return f4(0.f);
    const float4 E = e_adj(S, cx + 1, x, r);
    const float4 cf = S.coef[cx + 1];
    if (!GEN || rg.f9(x, r)) return (-cf.y * inv) * (E + jsum(S, cx + 1));
    if (n > 0 && x >= 1) {
      const int sy = rg.ey_row(r);
      if (sy >= 0) return (p.cpml_c[rg.ey_ci(r)] * inv) * fma4(-cf.z, E, pey);
    }
    return f4(0.f);
  };
  // the E half's psi inputs of row r: this cell's y- and x-strip psi, and the
  // x-strip psi of the neighbour an edge lane recomputes
  struct EPsi {
    float4 pey, pex, pex_nb;
  };
  auto ld_epsi = [&](int r) { return EPsi{ld_pey(x, r), ld_pex(x, r), ld_pex(x_nb, r)}; };
  // the H half's psi inputs of row y: Hy at x and x-1, Hx at x
  struct HPsi {
    float4 phy, phy_l, phx;
  };
  auto ld_hpsi = [&](int y) { return HPsi{ld_phy(x, y), ld_phy(x - 1, y), ld_phx(y)}; };
  // E half of this cell in row r of the segment: writes the new adjoint J and
  // E psi, adds the gradients; every lane of the warp must call it.
  auto e_half = [&](const St& S, int r, const EPsi& ep) {
    AdjE o{f4(0.f), f4(0.f), f4(0.f), f4(0.f)};
    float gv[KG];
#pragma unroll
    for (int k = 0; k < KG; ++k) gv[k] = 0.f;
    const bool f9 = active && (!GEN || rg.f9(x, r));
    if (active) {
      const float4 E = e_adj(S, cx + 1, x, r);
      const float4 cf = S.coef[cx + 1];
      o.elin = E;
      if (f9) {
        // E1 = ca E + cb/dx (cY - cX) - cb sum(gamma J);  J' = k1 J + k2 (E1 - E)/dt
        float4 e1 = S.e1[me];
        if ((src_own >> (r - rs)) & 1) {  // the forward added the source after E1
          const float w = __ldg(p.waveform + step);
          for (int s = 4 * lane_g; s < 4 * lane_g + 4 && s < p.ntx; ++s)
            if (__ldg(p.src_xy + 2 * s) == x && __ldg(p.src_xy + 2 * s + 1) == r) add_comp(e1, s & 3, -w);
        }
        const float4 en = S.en[me];
        const float4 e1tot = E + jsum(S, cx + 1);
        float4 elin = cf.x * e1tot;
        const float4 dedt = (e1 - en) * f4(p.inv_dt);
#pragma unroll
        for (int q = 0; q < ND + NL; ++q) {
          const float4 kq = S.ade[q * H + cx + 1];
          const float4 jin = S.lj[(q * H + cx + 1) * L + lo];
          elin = fma4(-kq.y * p.inv_dt, jin, elin);
          const size_t ja = (q * plane + (size_t)r * nx + x) * L + lo;
          if (q < ND) {  // Debye: J' = k1 J + k2 dE/dt, E1 -= cb gamma J
            st4(a.j[par ^ 1] + (size_t)g * p.gs_j + ja, kq.x * jin - (cf.y * kq.z) * e1tot);
          } else {       // Lorentz: J' = k1 J + k3 Jp + k2 dE/dt, Jp' = J, E1 -= cb J
            const size_t jpa = ((q - ND) * plane + (size_t)r * nx + x) * L + lo;
            st4(a.j[par ^ 1] + (size_t)g * p.gs_j + ja, kq.x * jin + S.ljp[(q - ND) * CX * L + me] - cf.y * e1tot);
            st4(a.jp[par ^ 1] + (size_t)g * p.gs_jp + jpa, kq.z * jin);
          }
          gv[3 + 3 * q] = dot4(jin, dedt);
          if (q < ND && a.grad_tau) {  // k1 and gamma depend on tau alone
            const float4 jn = S.jn[q * CX * L + me];
            gv[2 + 3 * q] = dot4(jin, jn);
            gv[4 + 3 * q] = -cf.y * dot4(e1tot, jn);
          }
        }
        o.elin = elin;
        o.cy = (cf.y * inv) * e1tot;
        o.cx = (-cf.y * inv) * e1tot;
        gv[0] = dot4(e1tot, en);
        gv[1] = __fdividef(dot4(e1tot, e1 - cf.x * en), cf.y);
      } else if (GEN && n > 0) {
        // transposed E-CPML: PEY' = b PEY + c/dx cX, E -= dteps PEY';
        //                    PEX' = b PEX + c/dx cY, E += dteps PEX'
        const int sy = rg.ey_row(r);
        if (x >= 1 && sy >= 0) {
          const int ci = rg.ey_ci(r);
          const float4 tot = fma4(-cf.z, E, ep.pey);
          st4(a.psi_ezy[par ^ 1] + (size_t)g * p.gs_psi_y + ((size_t)sy * nx + x) * L + lo, p.cpml_b[ci] * tot);
          o.cx = (p.cpml_c[ci] * inv) * tot;
        }
        const int sx = rg.ex_col(x);
        if (r >= 1 && sx >= 0) {
          const int ci = rg.ex_ci(x);
          const float4 tot = fma4(cf.z, E, ep.pex);
          st4(a.psi_ezx[par ^ 1] + (size_t)g * p.gs_psi_x + ((size_t)r * 2 * n + sx) * L + lo, p.cpml_b[ci] * tot);
          o.cy = (p.cpml_c[ci] * inv) * tot;
        }
      }
    }
    // sum over the L lanes of the cell; lane k % L adds gradient k (each
    // address receives one add per launch, so the order is fixed)
    double* gw = a.g + ((size_t)g * plane + (size_t)r * nx + x) * KP;
#pragma unroll
    for (int k = 0; k < KG; ++k) {
      if (k >= 2 && (k - 2) % 3 != 1 && !a.grad_tau) continue;  // k1, gamma slots: warp-uniform skip
      const float v = lane_sum<L>(gv[k]);
      if (f9 && (k % L) == lo) atomicAdd(gw + k, (double)v);
    }
    if (lw < L || lw >= 32 - L) {
      const int dx = lw < L ? -1 : 1;
      if (x + dx >= 0 && x + dx < nx) o.cye = cy_at(S, cx + 1 + dx, x + dx, r, ep.pex_nb);
    }
    return o;
  };
  // H half of this cell in row y; every lane of the warp must call it.
  auto h_half = [&](const St& S, int y, const AdjE& c, float4 cx_up, float4& d_u, const HPsi& hp) {
    float4 cy_l = shfl_up4(c.cy, L), cy_r = shfl_down4(c.cy, L);
    if (lw < L) cy_l = c.cye;
    if (lw >= 32 - L) cy_r = c.cye;
    if (!active) return;
    const size_t at = ((size_t)y * nx + x) * L + lo;
    const HAdj ry = hy_adj<GEN>(p, rg, x, y, S.lhy[mh], c.cy, cy_r, hp.phy);
    const HAdj rx = hx_adj<GEN>(p, rg, x, y, S.lhx[me], c.cx, cx_up, hp.phx);
    st4(a.hy[par ^ 1] + gf + at, ry.tot);
    st4(a.hx[par ^ 1] + gf + at, rx.tot);
    if (GEN && ry.s >= 0)
      st4(a.psi_hy[par ^ 1] + (size_t)g * p.gs_psi_x + ((size_t)y * 2 * n + ry.s) * L + lo, ry.psi);
    if (GEN && rx.s >= 0) st4(a.psi_hx[par ^ 1] + (size_t)g * p.gs_psi_y + ((size_t)rx.s * nx + x) * L + lo, rx.psi);
    float4 e = c.elin - ry.u - rx.u + d_u;
    if (!GEN || x >= 1) e = e + hy_adj<GEN>(p, rg, x - 1, y, S.lhy[mh - L], cy_l, c.cy, hp.phy_l).u;
    st4(a.ez[par ^ 1] + gf + at, e);
    d_u = rx.u;
  };

  if (!wait(0)) return;
  int k = 0;
  AdjE c;
  float4 d_u = f4(0.f);  // adjoint of E(x, y) - E(x, y-1) from the Hx update of the row below
  if (y0 > 0) {          // slot 0 holds row y0-1
    const float4 pey_b = ld_pey(x, y0 - 1), phx_b = ld_phx(y0 - 1);
    const EPsi ep0 = ld_epsi(y0);
    const float4 pcx = cx_row(st[0], y0 - 1, pey_b);
    if (!wait(1)) return;
    c = e_half(st[1 % NS], y0, ep0);
    if (active) d_u = hx_adj<GEN>(p, rg, x, y0 - 1, st[0].lhx[me], pcx, c.cx, phx_b).u;
    release(0);
    k = 1;
  } else {
    c = e_half(st[0], y0, ld_epsi(y0));
  }
  for (int y = y0; y < y1; ++y, ++k) {
    const bool has_up = k + 1 < nslots;
    // this iteration's psi inputs, issued before the wait and every store
    const HPsi hp = ld_hpsi(y);
    EPsi ep{f4(0.f), f4(0.f), f4(0.f)};
    if (y + 1 < y1) ep = ld_epsi(y + 1);
    else if (has_up) ep.pey = ld_pey(x, y + 1);
    if (has_up && !wait(k + 1)) return;
    AdjE up{f4(0.f), f4(0.f), f4(0.f), f4(0.f)};
    if (y + 1 < y1) up = e_half(st[(k + 1) % NS], y + 1, ep);
    else if (has_up) up.cx = cx_row(st[(k + 1) % NS], y + 1, ep.pey);
    h_half(st[k % NS], y, c, up.cx, d_u, hp);
    c = up;
    release(k);
  }
  if (k < nslots) release(k);  // the row above the segment
}

// ------------------------------------------------------------------------
// Consumer of interior tiles: every own cell, the halo columns x0-1 and
// x0+CX and the rows y0-1 and y1 lie in the interior E region, off the edges
// and outside every CPML strip, so the transposed step has no region tests
// and reduces to
//   mu = adj(E') + sum_q (k2_q/dt) adj(J_q')          (pointwise)
//   nu = cb/dx mu
//   adj(Hy) = adj(Hy') + nu(x) - nu(x+1),  adj(Hx) = adj(Hx') - nu(y) + nu(y+1)
//   adj(E)  = ca mu - sum_q (k2_q/dt) adj(J_q')
//             + db/dx (adj(Hy)(x-1) - adj(Hy)(x) + adj(Hx)(y) - adj(Hx)(y-1))
//   adj(J_q) = k1_q adj(J_q') - cb gamma_q mu
// with the operations of adj_consume in the same order.  Per row y a thread
// forms mu of its own cell in row y+1 (carried into the next row with nu),
// nu of the two neighbour cells in row y from the halo'd slices (no
// shuffles, no divergent edge lanes), the three H adjoints it needs (adj(Hx)
// of the row below is carried), and the new E adjoint, currents and
// gradients of its cell.
// ------------------------------------------------------------------------
template <int L, int ND, int NL>
CEEP_D void adj_consume_lean(const Adjoint2dParams& a, AdjStage<L, ND, NL>* st, uint64_t* full, uint64_t* empty,
                             int step, int par, int x0, int y0, int y1, int rs, int nslots, int g) {
  using St = AdjStage<L, ND, NL>;
  constexpr int CX = St::CX, H = St::H, NS = adj_stages<L, ND, NL>();
  constexpr int KG = 2 + 3 * (ND + NL), KP = adjoint2d_grad_width(ND + NL);
  const Fdtd2dParams& p = a.f;
  const int nx = p.nx;
  const int cx = threadIdx.x / L, lo = threadIdx.x % L;
  const int x = x0 + cx;
  const int lw = threadIdx.x & 31;
  const int lane_g = g * L + lo;
  const float inv = p.inv_dx, idt = p.inv_dt, dbdx = p.db_dx;
  const size_t plane = (size_t)nx * p.ny, gf = (size_t)g * p.gs_field;
  const int me = cx * L + lo;        // this cell in the plain slices
  const int mh = (cx + 1) * L + lo;  // this cell in the halo'd slices
  float4* ez_out = a.ez[par ^ 1] + gf;
  float4* hx_out = a.hx[par ^ 1] + gf;
  float4* hy_out = a.hy[par ^ 1] + gf;
  float4* j_out = a.j[par ^ 1] + (size_t)g * p.gs_j;
  float4* jp_out = a.jp[par ^ 1] + (size_t)g * p.gs_jp;

  // probe rows of the columns x-1, x, x+1 and this lane's source rows among
  // the slots' rows rs .. rs + nslots - 1 (<= 64), as bit masks
  uint64_t prb_l = 0, prb_c = 0, prb_r = 0, src_own = 0;
  for (int q = 0; q < p.nprobe; ++q) {
    const int px = __ldg(p.prb_xy + 2 * q), py = __ldg(p.prb_xy + 2 * q + 1) - rs;
    if (py >= 0 && py < nslots) {
      if (px == x - 1) prb_l |= 1ull << py;
      if (px == x) prb_c |= 1ull << py;
      if (px == x + 1) prb_r |= 1ull << py;
    }
  }
  for (int s = 4 * lane_g; s < 4 * lane_g + 4 && s < p.ntx; ++s) {
    const int sx = __ldg(p.src_xy + 2 * s), sy = __ldg(p.src_xy + 2 * s + 1) - rs;
    if (sx == x && sy >= 0 && sy < nslots) src_own |= 1ull << sy;
  }
  auto wait = [&](int k) {
    const bool ok = mbar_wait_bounded(&full[k % NS], (k / NS) & 1, kAdjWaitNs);
    if (__any_sync(0xffffffffu, !ok)) {
      if (lw == 0) adj_status(p.status, CEEP_ERR_TIMEOUT);
      return false;
    }
    return true;
  };
  auto release = [&](int k) {
    __syncwarp();
    if (lw == 0) mbar_arrive(&empty[k % NS]);
  };
  // mu of halo'd cell i (cell xc) of row r, probe gradient included
  auto mu_at = [&](const St& S, int i, int xc, int r, uint64_t mask) {
    float4 E = S.le[i * L + lo];
    if ((mask >> (r - rs)) & 1) inject_probes(a, E, xc, r, lane_g, step);
    float4 js = f4(0.f);
#pragma unroll
    for (int q = 0; q < ND + NL; ++q) js = fma4(S.ade[q * H + i].y * idt, S.lj[(q * H + i) * L + lo], js);
    return E + js;
  };
  auto nu_of = [&](const St& S, int i, float4 mu) { return (S.coef[i].y * inv) * mu; };

  // slot 0: row y0-1 (its adj(Hx) only), slot 1: row y0
  if (!wait(0)) return;
  if (!wait(1)) return;
  float4 mu_c = mu_at(st[1], cx + 1, x, y0, prb_c);
  float4 nu_c = nu_of(st[1], cx + 1, mu_c);
  float4 d_u;  // -db/dx adj(Hx)(x, y-1)
  {
    const St& B = st[0];
    const float4 nu_b = nu_of(B, cx + 1, mu_at(B, cx + 1, x, y0 - 1, prb_c));
    d_u = (-dbdx) * (B.lhx[me] - nu_b + nu_c);
  }
  release(0);
  int k = 1;
  for (int y = y0; y < y1; ++y, ++k) {
    if (!wait(k + 1)) return;  // row y+1 (row y1 < ny exists for an interior tile)
    const St& A = st[k % NS];
    const St& U = st[(k + 1) % NS];
    const float4 mu_u = mu_at(U, cx + 1, x, y + 1, prb_c);
    const float4 nu_u = nu_of(U, cx + 1, mu_u);
    const float4 nu_l = nu_of(A, cx, mu_at(A, cx, x - 1, y, prb_l));
    const float4 nu_r = nu_of(A, cx + 2, mu_at(A, cx + 2, x + 1, y, prb_r));
    const float4 hyt = A.lhy[mh] + nu_c - nu_r;
    const float4 hyt_l = A.lhy[mh - L] + nu_l - nu_c;
    const float4 hxt = A.lhx[me] - nu_c + nu_u;
    const size_t at = ((size_t)y * nx + x) * L + lo;
    st4(hy_out + at, hyt);
    st4(hx_out + at, hxt);

    // pointwise part: E adjoint, currents, gradients of this cell
    const float4 cf = A.coef[cx + 1];
    float4 e1 = A.e1[me];
    if ((src_own >> (y - rs)) & 1) {  // the forward added the source after E1
      const float w = __ldg(p.waveform + step);
      for (int s = 4 * lane_g; s < 4 * lane_g + 4 && s < p.ntx; ++s)
        if (__ldg(p.src_xy + 2 * s) == x && __ldg(p.src_xy + 2 * s + 1) == y) add_comp(e1, s & 3, -w);
    }
    const float4 en = A.en[me];
    const float4 dedt = (e1 - en) * f4(idt);
    float gv[KG];
#pragma unroll
    for (int kk = 0; kk < KG; ++kk) gv[kk] = 0.f;
    float4 elin = cf.x * mu_c;
#pragma unroll
    for (int q = 0; q < ND + NL; ++q) {
      const float4 kq = A.ade[q * H + cx + 1];
      const float4 jin = A.lj[(q * H + cx + 1) * L + lo];
      elin = fma4(-kq.y * idt, jin, elin);
      if (q < ND) {  // Debye
        st4(j_out + (q * plane + (size_t)y * nx + x) * L + lo, kq.x * jin - (cf.y * kq.z) * mu_c);
      } else {       // Lorentz (gamma = 1, second level J_prev)
        st4(j_out + (q * plane + (size_t)y * nx + x) * L + lo,
            kq.x * jin + A.ljp[(q - ND) * CX * L + me] - cf.y * mu_c);
        st4(jp_out + ((q - ND) * plane + (size_t)y * nx + x) * L + lo, kq.z * jin);
      }
      gv[3 + 3 * q] = dot4(jin, dedt);
      if (q < ND && a.grad_tau) {  // k1 and gamma depend on tau alone
        const float4 jn = A.jn[q * CX * L + me];
        gv[2 + 3 * q] = dot4(jin, jn);
        gv[4 + 3 * q] = -cf.y * dot4(mu_c, jn);
      }
    }
    gv[0] = dot4(mu_c, en);
    gv[1] = __fdividef(dot4(mu_c, e1 - cf.x * en), cf.y);
    float4 e = elin - dbdx * hyt - (-dbdx) * hxt + d_u;
    e = e + dbdx * hyt_l;
    st4(ez_out + at, e);
    d_u = (-dbdx) * hxt;

    double* gw = a.g + ((size_t)g * plane + (size_t)y * nx + x) * KP;
#pragma unroll
    for (int kk = 0; kk < KG; ++kk) {
      if (kk >= 2 && (kk - 2) % 3 != 1 && !a.grad_tau) continue;  // k1, gamma slots: warp-uniform skip
      const float v = lane_sum<L>(gv[kk]);
      if ((kk % L) == lo) atomicAdd(gw + kk, (double)v);
    }
    mu_c = mu_u;
    nu_c = nu_u;
    release(k);
  }
  release(k);  // the row above the segment
}

template <int L, int ND, int NL>
__global__ void __launch_bounds__(kAdjConsumers + 32, CEEP_ADJ_MIN_BLOCKS)
    adjoint2d_step_kernel(const Adjoint2dParams a, int step, int par, const float4* __restrict__ ez_n,
                          const float4* __restrict__ ez_np1, const float4* __restrict__ j_n) {
  extern __shared__ __align__(128) unsigned char smem_raw[];
  using St = AdjStage<L, ND, NL>;
  constexpr int NS = adj_stages<L, ND, NL>(), CX = St::CX;
  St* st = reinterpret_cast<St*>(smem_raw);
  uint64_t* full = reinterpret_cast<uint64_t*>(smem_raw + NS * sizeof(St));
  uint64_t* empty = full + NS;
  const int nx = a.f.nx, ny = a.f.ny, n = a.f.n;
  int bx, by;
  tile_frame_first(blockIdx.x, (nx + CX - 1) / CX, (ny + a.rows - 1) / a.rows, a.frame[0], a.frame[1], a.frame[2],
                   a.frame[3], bx, by);
  const int x0 = bx * CX, y0 = by * a.rows, g = blockIdx.y;
  const int y1 = min(y0 + a.rows, ny);
  const int rs = y0 > 0 ? y0 - 1 : 0;
  const int nslots = (y1 - rs) + (y1 < ny ? 1 : 0);
  if (threadIdx.x == 0) {
#pragma unroll
    for (int s = 0; s < NS; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], kAdjConsumers / 32);
    }
    mbar_init_fence();
  }
  __syncthreads();
  // Programmatic dependent launch, as in the forward step: every access to
  // adjoint state comes after the wait for the previous step's grid.
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
  if (threadIdx.x >= kAdjConsumers) {
    if (threadIdx.x == kAdjConsumers)
      adj_produce<L, ND, NL>(a, st, full, empty, par, ez_n, ez_np1, j_n, x0, y0, y1, rs, nslots, g);
    return;
  }
  // Block-uniform: own cells, the halo cells x0-1 and x0+CX and the rows
  // y0-1 and y1 all lie in the interior E region, off the edges, and the own
  // cells (and x0-1) in the plain H interior.
  const int m = n > 1 ? n : 1;
  const bool interior = x0 >= n + 2 && x0 + CX + 1 <= nx - m && y0 >= n + 2 && y1 + 1 <= ny - m;
  if (interior)
    adj_consume_lean<L, ND, NL>(a, st, full, empty, step, par, x0, y0, y1, rs, nslots, g);
  else
    adj_consume<L, ND, NL, true>(a, st, full, empty, step, par, x0, y0, y1, rs, nslots, g);
}

// ------------------------------------------------------------------------
// Host side
// ------------------------------------------------------------------------
// Tiles cost unequal time (CPML strips, probe rows), so a launch is cut into
// about three waves of tiles, frame tiles started first, for the block
// scheduler to balance; segments stay >= 8 rows so the two neighbour rows
// each one recomputes stay a small overhead.
static int adjoint2d_rows(int nx, int ny, int groups, int cells_per_block, long slots) {
  const long xb = (nx + cells_per_block - 1) / cells_per_block;
  for (int rows = kAdjMaxRows; rows > 8; --rows)
    if (xb * ((ny + rows - 1) / rows) * groups >= 3 * slots) return rows;
  return 8;
}

// Frame tile counts (left, right, top, bottom) of the adjoint's tile grid,
// by the kernel's own interior test: the leading and trailing columns and
// rows of tiles that are not interior.
static void adjoint_frame_counts(Adjoint2dParams& a, int cw) {
  const int n = a.f.n, m = n > 1 ? n : 1, nx = a.f.nx, ny = a.f.ny;
  const int gx = (nx + cw - 1) / cw, gy = (ny + a.rows - 1) / a.rows;
  auto in_x = [&](int bx) { const int x0 = bx * cw; return x0 >= n + 2 && x0 + cw + 1 <= nx - m; };
  auto in_y = [&](int by) {
    const int y0 = by * a.rows, y1 = y0 + a.rows < ny ? y0 + a.rows : ny;
    return y0 >= n + 2 && y1 + 1 <= ny - m;
  };
  int fl = 0, fr = 0, ft = 0, fb = 0;
  while (fl < gx && !in_x(fl)) ++fl;
  while (fr < gx - fl && !in_x(gx - 1 - fr)) ++fr;
  while (ft < gy && !in_y(ft)) ++ft;
  while (fb < gy - ft && !in_y(gy - 1 - fb)) ++fb;
  a.frame[0] = fl; a.frame[1] = fr; a.frame[2] = ft; a.frame[3] = fb;
}

template <int L, int ND, int NL>
static cudaError_t configure_l(Adjoint2dParams& a) {
  constexpr size_t smem = adj_smem_bytes<L, ND, NL>();
  auto kern = adjoint2d_step_kernel<L, ND, NL>;
  cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) return e;
  a.smem = (int)smem;
  if (a.rows > kAdjMaxRows) a.rows = kAdjMaxRows;
  if (a.rows <= 0) {
    int dev = 0, sms = 148, per_sm = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kAdjConsumers + 32, smem);
    if (e != cudaSuccess) return e;
    a.rows = adjoint2d_rows(a.f.nx, a.f.ny, a.f.groups, kAdjConsumers / L, (long)sms * (per_sm < 1 ? 1 : per_sm));
  }
  adjoint_frame_counts(a, kAdjConsumers / L);
  return cudaSuccess;
}

template <int L, int ND, int NL>
static cudaError_t launch_l(const Adjoint2dParams& a, int step, int par, const float4* ez_n, const float4* ez_np1,
                            const float4* j_n, cudaStream_t s) {
  constexpr int CX = kAdjConsumers / L;
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(((a.f.nx + CX - 1) / CX) * ((a.f.ny + a.rows - 1) / a.rows), a.f.groups);
  cfg.blockDim = dim3(kAdjConsumers + 32);
  cfg.dynamicSmemBytes = a.smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, adjoint2d_step_kernel<L, ND, NL>, a, step, par, ez_n, ez_np1, j_n);
}

template <int ND, int NL>
static cudaError_t dispatch_l(Adjoint2dParams& a, int step, int par, const float4* ez_n, const float4* ez_np1,
                              const float4* j_n, cudaStream_t s, bool configure) {
  switch (a.f.L) {
    case 1: return configure ? configure_l<1, ND, NL>(a) : launch_l<1, ND, NL>(a, step, par, ez_n, ez_np1, j_n, s);
    case 2: return configure ? configure_l<2, ND, NL>(a) : launch_l<2, ND, NL>(a, step, par, ez_n, ez_np1, j_n, s);
    case 4: return configure ? configure_l<4, ND, NL>(a) : launch_l<4, ND, NL>(a, step, par, ez_n, ez_np1, j_n, s);
    default: return configure ? configure_l<8, ND, NL>(a) : launch_l<8, ND, NL>(a, step, par, ez_n, ez_np1, j_n, s);
  }
}

static cudaError_t dispatch(Adjoint2dParams& a, int step, int par, const float4* ez_n, const float4* ez_np1,
                            const float4* j_n, cudaStream_t s, bool configure) {
  switch (a.f.n_debye * 3 + a.f.n_lorentz) {
    case 0: return dispatch_l<0, 0>(a, step, par, ez_n, ez_np1, j_n, s, configure);
    case 1: return dispatch_l<0, 1>(a, step, par, ez_n, ez_np1, j_n, s, configure);
    case 2: return dispatch_l<0, 2>(a, step, par, ez_n, ez_np1, j_n, s, configure);
    case 3: return dispatch_l<1, 0>(a, step, par, ez_n, ez_np1, j_n, s, configure);
    case 4: return dispatch_l<1, 1>(a, step, par, ez_n, ez_np1, j_n, s, configure);
    case 6: return dispatch_l<2, 0>(a, step, par, ez_n, ez_np1, j_n, s, configure);
    default: return cudaErrorInvalidValue;
  }
}

cudaError_t adjoint2d_configure(Adjoint2dParams& a) {
  return dispatch(a, 0, 0, nullptr, nullptr, nullptr, nullptr, true);
}

cudaError_t adjoint2d_launch_step(const Adjoint2dParams& a, int step, int par, const float4* ez_n,
                                  const float4* ez_np1, const float4* j_n, cudaStream_t s) {
  Adjoint2dParams q = a;
  return dispatch(q, step, par, ez_n, ez_np1, j_n, s, false);
}

}  // namespace ceep

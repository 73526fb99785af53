// extern "C" entry points declared in include/ceep_b200.h.
#include <cuda_runtime.h>

#include <cstdarg>
#include <cstdio>
#include <map>
#include <new>
#include <tuple>
#include <utility>

#include "../../include/ceep_b200.h"
#include "capi_internal.h"
#include "fdtd2d.cuh"
#include "common.cuh"

namespace {
thread_local char g_err[512] = "";
}

namespace ceep {
int fail(int code, const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
  return code;
}
int cuda_fail(cudaError_t e, const char* what) {
  return fail(CEEP_ERR_CUDA, "%s: %s", what, cudaGetErrorString(e));
}
}  // namespace ceep

using ceep::fail;

extern "C" int ceep_version(void) { return 100; }
extern "C" const char* ceep_last_error(void) { return g_err; }

// --------------------------------------------------------------------------
// 2D plan
// --------------------------------------------------------------------------
struct ceep2d_plan {
  ceep::Fdtd2dParams p;
  int cur = 0;       // ping-pong buffer holding the current state
  int tblock = 1;    // steps per launch (1, or 2 with the temporal-block kernel)
  int sentinel = 0;  // NaN/Inf check every this many steps (0: only at the end of each run range)
  ceep::Fdtd2dSide side{nullptr, nullptr, nullptr};  // the two-step frame tiles' stream
  // captured step loops keyed by (step0, nsteps, starting buffer, save buffers, save base, steps per launch)
  std::map<std::tuple<int64_t, int64_t, int, const void*, const void*, int64_t, int>, cudaGraphExec_t> graphs;
};

extern "C" int ceep2d_plan_create(const ceep2d_desc* d, ceep2d_plan** out) {
  if (!d || !out) return fail(CEEP_ERR_INVALID, "ceep2d_plan_create: null argument");
  *out = nullptr;
  const int n = d->cpml;
  if (d->nx < 3 || d->ny < 3) return fail(CEEP_ERR_INVALID, "grid %dx%d too small", d->nx, d->ny);
  if (n == 1 || n < 0) return fail(CEEP_ERR_INVALID, "cpml thickness must be 0 or >= 2 (got %d)", n);
  if (d->nx < 2 * n + 2 || d->ny < 2 * n + 2)
    return fail(CEEP_ERR_INVALID, "grid %dx%d must exceed twice the CPML (%d) by 2", d->nx, d->ny, n);
  if (d->ntx < 1 || d->ntx_pad < d->ntx || d->ntx_pad % 4)
    return fail(CEEP_ERR_INVALID, "ntx=%d ntx_pad=%d (pad must be a multiple of 4 and >= ntx)", d->ntx,
                d->ntx_pad);
  const int lanes = d->ntx_pad / 4;
  const int L = lanes <= 8 ? lanes : 8;
  if (lanes > 8 && lanes % 8)
    return fail(CEEP_ERR_INVALID, "ntx_pad=%d above 32 must be a multiple of 32", d->ntx_pad);
  if (L != 1 && L != 2 && L != 4 && L != 8)
    return fail(CEEP_ERR_INVALID, "ntx_pad=%d: pad to 4, 8, 16 or a multiple of 32", d->ntx_pad);
  if (d->n_debye < 0 || d->n_lorentz < 0 || d->n_debye + d->n_lorentz > 2)
    return fail(CEEP_ERR_UNSUPPORTED, "ADE poles: at most 2 per cell (debye=%d lorentz=%d)", d->n_debye,
                d->n_lorentz);
  if (d->nsteps < 1 || d->nprobe < 0) return fail(CEEP_ERR_INVALID, "nsteps/nprobe");
  for (int k = 0; k < 2; ++k)
    if (!d->ez[k] || !d->hx[k] || !d->hy[k]) return fail(CEEP_ERR_INVALID, "null field buffer");
  for (int k = 0; k < 2; ++k) {
    if (n > 0 && (!d->psi_hx[k] || !d->psi_hy[k] || !d->psi_ezx[k] || !d->psi_ezy[k] || !d->cpml_b || !d->cpml_c))
      return fail(CEEP_ERR_INVALID, "null CPML buffer");
    if (d->n_debye + d->n_lorentz > 0 && (!d->j[k] || !d->ade_coef || (d->n_lorentz && !d->j_prev[k])))
      return fail(CEEP_ERR_INVALID, "null ADE buffer");
  }
  if (!d->coef || !d->src_xy || !d->row_flags || !d->waveform || (d->nprobe && (!d->prb_xy || !d->probes)))
    return fail(CEEP_ERR_INVALID, "null coefficient/source/probe buffer");

  ceep2d_plan* pl = new (std::nothrow) ceep2d_plan();
  if (!pl) return fail(CEEP_ERR_INVALID, "host allocation failed");
  ceep::Fdtd2dParams& p = pl->p;
  p.nx = d->nx; p.ny = d->ny; p.n = n;
  p.ntx = d->ntx; p.L = L; p.groups = lanes / L;
  p.nprobe = d->nprobe; p.nsteps = d->nsteps;
  p.n_debye = d->n_debye; p.n_lorentz = d->n_lorentz;
  p.rows = d->rows_per_block > 0 ? d->rows_per_block : 0;
  p.rows_fixed = p.rows;
  p.db = d->db; p.db_dx = d->db * d->inv_dx; p.inv_dx = d->inv_dx; p.dt = d->dt;
  p.inv_dt = (float)(1.0 / (double)d->dt);
  const long long cells = (long long)d->nx * d->ny;
  const int np = d->n_debye + d->n_lorentz;
  p.gs_field = cells * L;
  p.gs_psi_x = (long long)d->ny * 2 * (n > 0 ? n : 1) * L;
  p.gs_psi_y = (long long)2 * (n > 0 ? n : 1) * d->nx * L;
  p.gs_j = cells * np * L;
  p.gs_jp = cells * d->n_lorentz * L;
  for (int k = 0; k < 2; ++k) {
    p.ez[k] = reinterpret_cast<float4*>(d->ez[k]);
    p.hx[k] = reinterpret_cast<float4*>(d->hx[k]);
    p.hy[k] = reinterpret_cast<float4*>(d->hy[k]);
    p.psi_hy[k] = reinterpret_cast<float4*>(d->psi_hy[k]);
    p.psi_hx[k] = reinterpret_cast<float4*>(d->psi_hx[k]);
    p.psi_ezx[k] = reinterpret_cast<float4*>(d->psi_ezx[k]);
    p.psi_ezy[k] = reinterpret_cast<float4*>(d->psi_ezy[k]);
    p.j[k] = reinterpret_cast<float4*>(d->j[k]);
    p.j_prev[k] = reinterpret_cast<float4*>(d->j_prev[k]);
  }
  p.coef = d->coef; p.ade_coef = d->ade_coef;
  p.cpml_b = d->cpml_b; p.cpml_c = d->cpml_c;
  p.src_xy = d->src_xy; p.prb_xy = d->prb_xy; p.row_flags = d->row_flags;
  p.waveform = d->waveform; p.probes = d->probes;
  p.status = d->status;
  p.fault_row = -1;
  p.wait_ns = 1000000000ull;
  p.split2 = 0;
  cudaError_t ce = ceep::fdtd2d_configure(p);
  if (ce != cudaSuccess) {
    delete pl;
    return ceep::cuda_fail(ce, "fdtd2d_configure");
  }
  // the frame tiles' stream at the highest priority, so that their blocks
  // (few, long) start first and the interior kernel's fill the rest
  int least = 0, greatest = 0;
  ce = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (ce == cudaSuccess) ce = cudaStreamCreateWithPriority(&pl->side.stream, cudaStreamNonBlocking, greatest);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&pl->side.fork, cudaEventDisableTiming);
  if (ce == cudaSuccess) ce = cudaEventCreateWithFlags(&pl->side.join, cudaEventDisableTiming);
  if (ce != cudaSuccess) {
    ceep2d_plan_destroy(pl);
    return ceep::cuda_fail(ce, "ceep2d_plan_create: side stream");
  }
  *out = pl;
  return CEEP_OK;
}

// Launch steps [step0, step0 + nsteps): pairs through the two-step kernel when
// tblock == 2, the rest one step at a time.  Every launch reads buffer `cur`
// and writes the other.
static int64_t launch_count(int64_t nsteps, int tblock) { return tblock == 2 ? (nsteps + 1) / 2 : nsteps; }

// With a status word, the NaN/Inf sentinel scans the current Ez and the probe
// samples recorded since its previous scan after every `sentinel` steps (0:
// none in between) and after the range's last step.
static int run_steps(const ceep::Fdtd2dParams& p, int64_t step0, int64_t nsteps, int cur, int tblock, int sentinel,
                     cudaStream_t s, const ceep::Fdtd2dSide* side) {
  int64_t checked = step0;
  for (int64_t k = 0; k < nsteps;) {
    const bool two = tblock == 2 && k + 1 < nsteps;
    cudaError_t e = two ? ceep::fdtd2d_launch_step2(p, (int)(step0 + k), cur, s, side)
                        : ceep::fdtd2d_launch_step(p, (int)(step0 + k), cur, s);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "fdtd2d step launch");
    k += two ? 2 : 1;
    cur ^= 1;
    const int64_t done = step0 + k;
    if (p.status && (k == nsteps || (sentinel > 0 && done / sentinel != checked / sentinel))) {
      e = ceep::finite_check_launch(p.ez[cur], p.groups * p.gs_field, p.probes, p.ntx, p.nprobe, p.nsteps,
                                    (int)checked, (int)done, p.status, s);
      if (e != cudaSuccess) return ceep::cuda_fail(e, "finite_check_kernel launch");
      checked = done;
    }
  }
  return CEEP_OK;
}

// Captured step loops hold the kernel parameters of their capture: drop them
// when a setting that the launches carry changes.
static void drop_graphs(ceep2d_plan* pl) {
  for (auto& kv : pl->graphs) cudaGraphExecDestroy(kv.second);
  pl->graphs.clear();
}

static int plan_run(ceep2d_plan* pl, int64_t step0, int64_t nsteps, void* stream, int use_graph, float* save_ez,
                    float* save_j, int64_t save_base) {
  if (!pl) return fail(CEEP_ERR_INVALID, "null plan");
  if (step0 < 0 || nsteps < 0 || step0 + nsteps > pl->p.nsteps)
    return fail(CEEP_ERR_INVALID, "steps [%lld, %lld) outside [0, %d)", (long long)step0,
                (long long)(step0 + nsteps), pl->p.nsteps);
  if (save_ez && save_base > step0) return fail(CEEP_ERR_INVALID, "save buffers need save_base <= step0");
  if (nsteps == 0) return CEEP_OK;
  ceep::Fdtd2dParams q = pl->p;
  q.save_ez = reinterpret_cast<float4*>(save_ez);
  q.save_j = save_ez ? reinterpret_cast<float4*>(save_j) : nullptr;
  q.save_base = (int)save_base;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const int cur = pl->cur;
  const int cur_after = cur ^ (int)(launch_count(nsteps, pl->tblock) & 1);
  const ceep::Fdtd2dSide* side = pl->side.stream ? &pl->side : nullptr;
  if (!use_graph || s == nullptr) {
    int rc = run_steps(q, step0, nsteps, cur, pl->tblock, pl->sentinel, s, side);
    if (rc == CEEP_OK) pl->cur = cur_after;
    return rc;
  }
  auto key = std::make_tuple(step0, nsteps, cur, (const void*)save_ez, (const void*)q.save_j, save_base, pl->tblock);
  auto it = pl->graphs.find(key);
  if (it == pl->graphs.end()) {
    cudaGraph_t g;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "cudaStreamBeginCapture");
    int rc = run_steps(q, step0, nsteps, cur, pl->tblock, pl->sentinel, s, side);
    e = cudaStreamEndCapture(s, &g);
    if (rc != CEEP_OK) { if (e == cudaSuccess) cudaGraphDestroy(g); return rc; }
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

extern "C" int ceep2d_plan_run(ceep2d_plan* pl, int64_t step0, int64_t nsteps, void* stream, int use_graph) {
  return plan_run(pl, step0, nsteps, stream, use_graph, nullptr, nullptr, 0);
}

extern "C" int ceep2d_plan_run_save(ceep2d_plan* pl, int64_t step0, int64_t nsteps, void* stream, int use_graph,
                                    float* save_ez, float* save_j, int64_t save_base) {
  if (!save_ez) return fail(CEEP_ERR_INVALID, "ceep2d_plan_run_save: null save buffer");
  return plan_run(pl, step0, nsteps, stream, use_graph, save_ez, save_j, save_base);
}

extern "C" int ceep2d_plan_set_current_buffer(ceep2d_plan* pl, int cur) {
  if (!pl || (cur != 0 && cur != 1)) return fail(CEEP_ERR_INVALID, "bad plan or buffer index");
  pl->cur = cur;
  return CEEP_OK;
}

extern "C" int ceep2d_plan_current_buffer(const ceep2d_plan* pl) { return pl ? pl->cur : -1; }
extern "C" int ceep2d_plan_reset(ceep2d_plan* pl) {
  if (!pl) return fail(CEEP_ERR_INVALID, "null plan");
  pl->cur = 0;
  return CEEP_OK;
}
extern "C" int64_t ceep2d_desc_size(void) { return (int64_t)sizeof(ceep2d_desc); }
extern "C" int ceep2d_plan_rows(const ceep2d_plan* pl) { return pl ? pl->p.rows : 0; }

extern "C" int ceep2d_plan_destroy(ceep2d_plan* pl) {
  if (!pl) return CEEP_OK;
  for (auto& kv : pl->graphs) cudaGraphExecDestroy(kv.second);
  if (pl->side.stream) cudaStreamSynchronize(pl->side.stream);
  if (pl->side.join) cudaEventDestroy(pl->side.join);
  if (pl->side.fork) cudaEventDestroy(pl->side.fork);
  if (pl->side.stream) cudaStreamDestroy(pl->side.stream);
  delete pl;
  return CEEP_OK;
}

extern "C" int ceep2d_plan_set_frame_split(ceep2d_plan* pl, int32_t on) {
  if (!pl) return fail(CEEP_ERR_INVALID, "null plan");
  if (pl->p.split2 != (on != 0)) drop_graphs(pl);
  pl->p.split2 = on != 0;
  return CEEP_OK;
}

extern "C" int ceep2d_launches_per_step(const ceep2d_plan* pl) { return pl ? 1 : 0; }

extern "C" int ceep2d_plan_set_temporal_block(ceep2d_plan* pl, int steps) {
  if (!pl) return fail(CEEP_ERR_INVALID, "null plan");
  if (steps != 1 && steps != 2) return fail(CEEP_ERR_INVALID, "temporal block of %d steps (1 or 2)", steps);
  pl->tblock = steps;
  return CEEP_OK;
}

extern "C" int ceep2d_plan_temporal_block(const ceep2d_plan* pl) { return pl ? pl->tblock : 0; }

extern "C" int ceep2d_plan_set_sentinel(ceep2d_plan* pl, int32_t interval) {
  if (!pl || interval < 0) return fail(CEEP_ERR_INVALID, "ceep2d_plan_set_sentinel: bad plan or interval %d", interval);
  if (interval != pl->sentinel) drop_graphs(pl);
  pl->sentinel = interval;
  return CEEP_OK;
}

extern "C" int ceep2d_plan_set_wait_limit(ceep2d_plan* pl, uint64_t ns) {
  if (!pl || ns == 0) return fail(CEEP_ERR_INVALID, "ceep2d_plan_set_wait_limit: bad plan or zero limit");
  if (ns != pl->p.wait_ns) drop_graphs(pl);
  pl->p.wait_ns = ns;
  return CEEP_OK;
}

extern "C" int ceep2d_plan_inject_copy_fault(ceep2d_plan* pl, int32_t row) {
  if (!pl || row < -1 || row >= pl->p.ny)
    return fail(CEEP_ERR_INVALID, "ceep2d_plan_inject_copy_fault: bad plan or row %d", row);
  if (row != pl->p.fault_row) drop_graphs(pl);
  pl->p.fault_row = row;
  return CEEP_OK;
}

extern "C" int64_t ceep2d_plan_launches(const ceep2d_plan* pl, int64_t nsteps) {
  if (!pl || nsteps < 0) return 0;
  // a split two-step launch is two kernels (frame tiles, interior tiles)
  const ceep::Fdtd2dParams& p = pl->p;
  const bool split = pl->side.stream && p.split2 && p.nframe2 > 0 && p.ntiles2 > p.nframe2;
  const int64_t pairs = pl->tblock == 2 ? nsteps / 2 : 0;
  return (nsteps - 2 * pairs) + pairs * (split ? 2 : 1);
}

// --------------------------------------------------------------------------
// 3D plan
// --------------------------------------------------------------------------
#include "fdtd3d.cuh"

struct ceep3d_plan {
  ceep::Fdtd3dParams p;
  std::map<std::tuple<int64_t, int64_t, const void*, int64_t, int>, cudaGraphExec_t> graphs;
  ceep::Fdtd3dSide side{nullptr, nullptr, nullptr};   // the H shell's stream
};

extern "C" int64_t ceep3d_desc_size(void) { return (int64_t)sizeof(ceep3d_desc); }

extern "C" int ceep3d_plan_create(const ceep3d_desc* d, ceep3d_plan** out) {
  if (!d || !out) return fail(CEEP_ERR_INVALID, "ceep3d_plan_create: null argument");
  *out = nullptr;
  const int n = d->cpml;
  if (n == 1 || n < 0) return fail(CEEP_ERR_INVALID, "cpml thickness must be 0 or >= 2 (got %d)", n);
  if (d->nx < 2 * n + 2 || d->ny < 2 * n + 2 || d->nz < 2 * n + 2 || d->nx < 3 || d->ny < 3 || d->nz < 3)
    return fail(CEEP_ERR_INVALID, "grid %dx%dx%d must exceed twice the CPML (%d) by 2", d->nx, d->ny, d->nz, n);
  if (d->ntx < 1 || d->ntx_pad < d->ntx || d->ntx_pad % 4)
    return fail(CEEP_ERR_INVALID, "ntx=%d ntx_pad=%d", d->ntx, d->ntx_pad);
  const int lanes = d->ntx_pad / 4;
  const int L = lanes <= 8 ? lanes : 8;
  if ((lanes > 8 && lanes % 8) || (L != 1 && L != 2 && L != 4 && L != 8))
    return fail(CEEP_ERR_INVALID, "ntx_pad=%d: pad to 4, 8, 16 or a multiple of 32", d->ntx_pad);
  if (d->n_debye < 0 || d->n_lorentz < 0 || d->n_debye + d->n_lorentz > 2)
    return fail(CEEP_ERR_UNSUPPORTED, "ADE poles: at most 2 per cell");
  if (d->nsteps < 1 || d->nprobe < 0) return fail(CEEP_ERR_INVALID, "nsteps/nprobe");
  if (!d->ex || !d->ey || !d->ez || !d->hx || !d->hy || !d->hz || !d->coef || !d->src_xyz || !d->waveform ||
      (d->nprobe && (!d->prb_xyz || !d->probes)))
    return fail(CEEP_ERR_INVALID, "null field/coefficient/source/probe buffer");
  if (n > 0 && (!d->psi_hxy || !d->psi_hzy || !d->psi_hyx || !d->psi_hzx || !d->psi_hxz || !d->psi_hyz ||
                !d->cpml_b || !d->cpml_c))
    return fail(CEEP_ERR_INVALID, "null CPML buffer");
  if (d->n_debye + d->n_lorentz > 0 && (!d->j || !d->ade_coef || (d->n_lorentz && !d->j_prev)))
    return fail(CEEP_ERR_INVALID, "null ADE buffer");
  ceep3d_plan* pl = new (std::nothrow) ceep3d_plan();
  if (!pl) return fail(CEEP_ERR_INVALID, "host allocation failed");
  ceep::Fdtd3dParams& p = pl->p;
  p.nx = d->nx; p.ny = d->ny; p.nz = d->nz; p.n = n;
  p.ntx = d->ntx; p.L = L; p.groups = lanes / L;
  p.nprobe = d->nprobe; p.nsteps = d->nsteps;
  p.n_debye = d->n_debye; p.n_lorentz = d->n_lorentz;
  p.zrows = d->z_rows > 0 ? d->z_rows : 16;
  p.zrows_shell = d->shell_z_rows > 0 ? d->shell_z_rows : 4;
  p.zsegs = (d->nz + p.zrows - 1) / p.zrows;
  const int nzi = d->nz - 2 * n - 1;
  p.zsegs_e = nzi > 0 ? (nzi + p.zrows - 1) / p.zrows : 0;
  p.inv_dx = d->inv_dx; p.dt = d->dt; p.inv_dt = (float)(1.0 / (double)d->dt);
  const long long cells = (long long)d->nx * d->ny * d->nz;
  const long long nn = n > 0 ? n : 1;
  p.gs_field = cells * L;
  p.gs_px = (long long)d->nz * d->ny * 2 * nn * L;
  p.gs_py = (long long)d->nz * 2 * nn * d->nx * L;
  p.gs_pz = 2 * nn * d->ny * (long long)d->nx * L;
  p.gs_j = cells * 3 * (d->n_debye + d->n_lorentz) * L;
  p.gs_jp = cells * 3 * d->n_lorentz * L;
  auto f4p = [](float* q) { return reinterpret_cast<float4*>(q); };
  p.ex = f4p(d->ex); p.ey = f4p(d->ey); p.ez = f4p(d->ez);
  p.hx = f4p(d->hx); p.hy = f4p(d->hy); p.hz = f4p(d->hz);
  p.psi_hxy = f4p(d->psi_hxy); p.psi_hzy = f4p(d->psi_hzy);
  p.psi_hyx = f4p(d->psi_hyx); p.psi_hzx = f4p(d->psi_hzx);
  p.psi_hxz = f4p(d->psi_hxz); p.psi_hyz = f4p(d->psi_hyz);
  p.j = f4p(d->j); p.j_prev = f4p(d->j_prev);
  p.coef = d->coef; p.ade_coef = d->ade_coef; p.cpml_b = d->cpml_b; p.cpml_c = d->cpml_c;
  p.src_xyz = d->src_xyz; p.prb_xyz = d->prb_xyz; p.waveform = d->waveform; p.probes = d->probes;
  p.save_e = nullptr;
  p.save_cs = p.groups * (long long)(d->nx - 2 * n - 1) * (d->ny - 2 * n - 1) * (d->nz - 2 * n - 1) * L;
  p.save_base = 0;
  p.interior_only = 0;
  // the H shell's stream at the highest priority, so that its blocks (few,
  // long, register-heavy) start first and the box's fill the rest
  int least = 0, greatest = 0;
  cudaError_t e = cudaDeviceGetStreamPriorityRange(&least, &greatest);
  if (e == cudaSuccess) e = cudaStreamCreateWithPriority(&pl->side.stream, cudaStreamNonBlocking, greatest);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pl->side.fork, cudaEventDisableTiming);
  if (e == cudaSuccess) e = cudaEventCreateWithFlags(&pl->side.join, cudaEventDisableTiming);
  if (e != cudaSuccess) {
    ceep3d_plan_destroy(pl);
    return ceep::cuda_fail(e, "ceep3d_plan_create: side stream");
  }
  *out = pl;
  return CEEP_OK;
}

static int run_steps3d(const ceep::Fdtd3dParams& q, int64_t step0, int64_t nsteps, cudaStream_t s,
                       const ceep::Fdtd3dSide* side) {
  for (int64_t k = 0; k < nsteps; ++k) {
    cudaError_t e = ceep::fdtd3d_launch_step(q, (int)(step0 + k), s, side);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "fdtd3d step launch");
  }
  return CEEP_OK;
}

static int plan_run3d(ceep3d_plan* pl, int64_t step0, int64_t nsteps, void* stream, int use_graph, float* save_e,
                      int64_t save_base, int interior_only) {
  if (!pl) return fail(CEEP_ERR_INVALID, "null plan");
  if (step0 < 0 || nsteps < 0 || step0 + nsteps > pl->p.nsteps)
    return fail(CEEP_ERR_INVALID, "steps [%lld, %lld) outside [0, %d)", (long long)step0,
                (long long)(step0 + nsteps), pl->p.nsteps);
  if (save_e && (save_base < 0 || save_base > step0))
    return fail(CEEP_ERR_INVALID, "save buffer needs 0 <= save_base <= step0");
  if (nsteps == 0) return CEEP_OK;
  ceep::Fdtd3dParams q = pl->p;
  q.save_e = reinterpret_cast<float4*>(save_e);
  q.save_base = save_e ? (int)save_base : 0;
  q.interior_only = interior_only && pl->p.n > 0 ? 1 : 0;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const ceep::Fdtd3dSide* side = pl->side.stream ? &pl->side : nullptr;
  if (!use_graph || s == nullptr) return run_steps3d(q, step0, nsteps, s, side);
  auto key = std::make_tuple(step0, nsteps, (const void*)save_e, (int64_t)q.save_base, q.interior_only);
  auto it = pl->graphs.find(key);
  if (it == pl->graphs.end()) {
    cudaGraph_t g;
    cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "cudaStreamBeginCapture");
    int rc = run_steps3d(q, step0, nsteps, s, side);
    e = cudaStreamEndCapture(s, &g);
    if (rc != CEEP_OK) { if (e == cudaSuccess) cudaGraphDestroy(g); return rc; }
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

extern "C" int ceep3d_plan_run(ceep3d_plan* pl, int64_t step0, int64_t nsteps, void* stream, int use_graph) {
  return plan_run3d(pl, step0, nsteps, stream, use_graph, nullptr, 0, 0);
}

extern "C" int ceep3d_plan_run_save(ceep3d_plan* pl, int64_t step0, int64_t nsteps, void* stream, int use_graph,
                                    float* save_e, int64_t save_base, int interior_only) {
  if (!save_e) return fail(CEEP_ERR_INVALID, "ceep3d_plan_run_save: null save buffer");
  return plan_run3d(pl, step0, nsteps, stream, use_graph, save_e, save_base, interior_only);
}

extern "C" int ceep3d_plan_destroy(ceep3d_plan* pl) {
  if (!pl) return CEEP_OK;
  for (auto& kv : pl->graphs) cudaGraphExecDestroy(kv.second);
  if (pl->side.stream) cudaStreamSynchronize(pl->side.stream);
  if (pl->side.join) cudaEventDestroy(pl->side.join);
  if (pl->side.fork) cudaEventDestroy(pl->side.fork);
  if (pl->side.stream) cudaStreamDestroy(pl->side.stream);
  delete pl;
  return CEEP_OK;
}

// --------------------------------------------------------------------------
// 2D adjoint
// --------------------------------------------------------------------------
#include "adjoint2d.cuh"

struct ceep2d_adjoint {
  ceep::Adjoint2dParams a;
  int cur = 0;
};

extern "C" int ceep2d_adjoint_create(const ceep2d_plan* plan, const ceep2d_adjoint_desc* d, ceep2d_adjoint** out) {
  if (!plan || !d || !out) return fail(CEEP_ERR_INVALID, "ceep2d_adjoint_create: null argument");
  *out = nullptr;
  for (int k = 0; k < 2; ++k) {
    if (!d->ez[k] || !d->hx[k] || !d->hy[k] || !d->grad)
      return fail(CEEP_ERR_INVALID, "adjoint: null state/gradient buffer");
    if (plan->p.n > 0 && (!d->psi_hx[k] || !d->psi_hy[k] || !d->psi_ezx[k] || !d->psi_ezy[k]))
      return fail(CEEP_ERR_INVALID, "adjoint: null psi buffer");
    if (plan->p.n_debye + plan->p.n_lorentz && !d->j[k]) return fail(CEEP_ERR_INVALID, "adjoint: null current buffer");
    if (plan->p.n_lorentz && !d->jp[k]) return fail(CEEP_ERR_INVALID, "adjoint: null Lorentz J_prev buffer");
  }
  if (plan->p.nprobe && !d->probe_grad) return fail(CEEP_ERR_INVALID, "adjoint: null probe gradient");
  ceep2d_adjoint* ad = new (std::nothrow) ceep2d_adjoint();
  if (!ad) return fail(CEEP_ERR_INVALID, "host allocation failed");
  ceep::Adjoint2dParams& a = ad->a;
  a.f = plan->p;
  a.rows = 0;
  auto f4p = [](float* q) { return reinterpret_cast<float4*>(q); };
  for (int k = 0; k < 2; ++k) {
    a.ez[k] = f4p(d->ez[k]);
    a.hx[k] = f4p(d->hx[k]);
    a.hy[k] = f4p(d->hy[k]);
    a.psi_hx[k] = f4p(d->psi_hx[k]);
    a.psi_hy[k] = f4p(d->psi_hy[k]);
    a.psi_ezx[k] = f4p(d->psi_ezx[k]);
    a.psi_ezy[k] = f4p(d->psi_ezy[k]);
    a.j[k] = f4p(d->j[k]);
    a.jp[k] = f4p(d->jp[k]);
  }
  a.g = d->grad;
  a.probe_grad = d->probe_grad;
  a.grad_tau = d->grad_tau ? 1 : 0;
  cudaError_t e = ceep::adjoint2d_configure(a);
  if (e != cudaSuccess) {
    delete ad;
    return ceep::cuda_fail(e, "adjoint2d configure");
  }
  *out = ad;
  return CEEP_OK;
}

extern "C" int ceep2d_adjoint_run(ceep2d_adjoint* ad, int64_t step_hi, int64_t nsteps, const float* seg_ez,
                                  const float* seg_j, int64_t seg_base, void* stream) {
  if (!ad || !seg_ez) return fail(CEEP_ERR_INVALID, "ceep2d_adjoint_run: null argument");
  const ceep::Fdtd2dParams& f = ad->a.f;
  if (nsteps < 0 || step_hi > f.nsteps || step_hi - nsteps < seg_base || (f.n_debye && ad->a.grad_tau && !seg_j))
    return fail(CEEP_ERR_INVALID, "ceep2d_adjoint_run: steps [%lld, %lld) with segment base %lld",
                (long long)(step_hi - nsteps), (long long)step_hi, (long long)seg_base);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t fslot = (size_t)f.groups * f.gs_field, jslot = (size_t)f.groups * f.gs_j;
  const float4* E = reinterpret_cast<const float4*>(seg_ez);
  const float4* J = reinterpret_cast<const float4*>(seg_j);
  for (int64_t n = step_hi - 1; n >= step_hi - nsteps; --n) {
    const size_t k = (size_t)(n - seg_base);
    cudaError_t e = ceep::adjoint2d_launch_step(ad->a, (int)n, ad->cur, E + k * fslot, E + (k + 1) * fslot,
                                                (J && ad->a.grad_tau) ? J + k * jslot : nullptr, s);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "adjoint2d step launch");
    ad->cur ^= 1;
  }
  return CEEP_OK;
}

extern "C" int ceep2d_adjoint_reset(ceep2d_adjoint* ad) {
  if (!ad) return fail(CEEP_ERR_INVALID, "null adjoint");
  ad->cur = 0;
  return CEEP_OK;
}

extern "C" int ceep2d_adjoint_destroy(ceep2d_adjoint* ad) {
  delete ad;
  return CEEP_OK;
}

extern "C" int64_t ceep2d_adjoint_desc_size(void) { return (int64_t)sizeof(ceep2d_adjoint_desc); }

// --------------------------------------------------------------------------
// 3D adjoint
// --------------------------------------------------------------------------
#include "adjoint3d.cuh"

struct ceep3d_adjoint {
  ceep::Adjoint3dParams a;
};

extern "C" int ceep3d_adjoint_create(const ceep3d_plan* plan, const ceep3d_adjoint_desc* d, ceep3d_adjoint** out) {
  if (!plan || !d || !out) return fail(CEEP_ERR_INVALID, "ceep3d_adjoint_create: null argument");
  *out = nullptr;
  const ceep::Fdtd3dParams& f = plan->p;
  if (f.n_lorentz) return fail(CEEP_ERR_UNSUPPORTED, "3D adjoint: Lorentz poles are not supported");
  if (f.n < 1) return fail(CEEP_ERR_UNSUPPORTED, "3D adjoint: needs a CPML of at least 2 cells");
  if (!d->mu || !d->nu || !d->grad || (f.n_debye && !d->lj))
    return fail(CEEP_ERR_INVALID, "3D adjoint: null state/gradient buffer");
  if (f.nprobe && !d->probe_grad) return fail(CEEP_ERR_INVALID, "3D adjoint: null probe gradient");
  ceep3d_adjoint* ad = new (std::nothrow) ceep3d_adjoint();
  if (!ad) return fail(CEEP_ERR_INVALID, "host allocation failed");
  ceep::Adjoint3dParams& a = ad->a;
  a.f = f;
  a.f.save_e = nullptr;
  const int eh = f.nz - 2 * f.n;  // H box [n, nz-n), E interior [n+1, nz-n)
  a.zsegs_h = (eh + f.zrows - 1) / f.zrows;
  a.zsegs_e = (eh - 1 + f.zrows - 1) / f.zrows;
  a.cs = (long long)f.groups * f.gs_field;
  a.icells = (long long)(f.nx - 2 * f.n - 1) * (f.ny - 2 * f.n - 1) * (f.nz - 2 * f.n - 1);
  a.ks = 2 + f.n_debye;
  a.mu = reinterpret_cast<float4*>(d->mu);
  a.nu = reinterpret_cast<float4*>(d->nu);
  a.lj = reinterpret_cast<float4*>(d->lj);
  a.g = d->grad;
  a.probe_grad = d->probe_grad;
  *out = ad;
  return CEEP_OK;
}

extern "C" int ceep3d_adjoint_run(ceep3d_adjoint* ad, int64_t step_hi, int64_t nsteps, const float* seg_e,
                                  int64_t seg_base, void* stream) {
  if (!ad || !seg_e) return fail(CEEP_ERR_INVALID, "ceep3d_adjoint_run: null argument");
  const ceep::Adjoint3dParams& a = ad->a;
  if (nsteps < 0 || step_hi > a.f.nsteps || step_hi - nsteps < seg_base || seg_base < 0)
    return fail(CEEP_ERR_INVALID, "ceep3d_adjoint_run: steps [%lld, %lld) with segment base %lld",
                (long long)(step_hi - nsteps), (long long)step_hi, (long long)seg_base);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t slot = 3 * (size_t)a.f.save_cs;   // interior E box per component
  const float4* E = reinterpret_cast<const float4*>(seg_e);
  for (int64_t n = step_hi - 1; n >= step_hi - nsteps; --n) {
    const size_t k = (size_t)(n - seg_base);
    cudaError_t e = ceep::adjoint3d_launch_step(a, (int)n, E + k * slot, E + (k + 1) * slot, n == seg_base, s);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "adjoint3d step launch");
  }
  return CEEP_OK;
}

extern "C" int32_t ceep3d_adjoint_grad_slots(const ceep3d_adjoint* ad) { return ad ? ad->a.ks : 0; }

extern "C" int ceep3d_adjoint_destroy(ceep3d_adjoint* ad) {
  delete ad;
  return CEEP_OK;
}

extern "C" int64_t ceep3d_adjoint_desc_size(void) { return (int64_t)sizeof(ceep3d_adjoint_desc); }

extern "C" int ceep2d_adjoint_rows(const ceep2d_adjoint* ad) { return ad ? ad->a.rows : 0; }

extern "C" int ceep2d_adjoint_set_rows(ceep2d_adjoint* ad, int32_t rows) {
  if (!ad || rows < 0) return fail(CEEP_ERR_INVALID, "ceep2d_adjoint_set_rows: bad adjoint or rows %d", rows);
  ad->a.rows = rows;  // 0: the automatic choice
  cudaError_t e = ceep::adjoint2d_configure(ad->a);
  return e == cudaSuccess ? CEEP_OK : ceep::cuda_fail(e, "adjoint2d configure");
}

#ifndef CEEP_PACK_FRAME_PIECES
#define CEEP_PACK_FRAME_PIECES 1  // blocks per frame tile in the packed two-step tables
#endif

// --------------------------------------------------------------------------
// Packed multi-phantom 2D launch
// --------------------------------------------------------------------------
#include <algorithm>
#include <vector>

namespace {
struct PackClass {
  int L, nd, nl;
  // One-step tiles: the frame tiles of every phantom (phantoms in order of
  // decreasing step count), then their interior tiles, so that the running
  // tiles of each part form a prefix and a launch starts every running
  // phantom's frame tiles (several times an interior tile's cost) first.
  ceep::PackTile* tiles;          // device (inside the caller's workspace)
  int nf = 0;                     // frame tiles; the interior part starts at tiles + nf
  std::vector<int> act_f, act_i;  // running frame / interior tiles at each step
  // two steps per launch: tiles of the two-step geometry, laid out the same
  // way; at pair t (steps 2t, 2t+1) the phantoms with >= 2t+2 steps run
  // two-step tiles (a prefix of each part) and those with exactly 2t+1 steps
  // run one-step tiles, a range of each part of the one-step table
  ceep::PackTile* tiles2;
  int nf2 = 0;
  std::vector<int> act2_f, act2_i, tail_f_lo, tail_f_hi, tail_i_lo, tail_i_hi;
};
size_t align16(size_t v) { return (v + 15) & ~(size_t)15; }
}  // namespace

struct ceep2d_pack {
  std::vector<ceep2d_plan*> plans;
  ceep::Fdtd2dParams* params = nullptr;  // device
  std::vector<PackClass> classes;
  int max_steps = 0;
  int tblock = 1;  // steps per launch (1 or 2)
  // Packing of the classes in time: 0 = one stream, the classes' launches
  // interleaved step by step (each launch waits for the previous class's);
  // 1 = one stream per class, so the classes' launch chains (independent
  // phantoms) run side by side, forked from and joined to the caller's stream.
  int concurrent = 0;
  std::vector<cudaStream_t> side;     // one per class beyond the first (concurrent packing)
  std::vector<cudaEvent_t> events;    // fork + one join per side stream
  std::map<std::tuple<int64_t, int64_t, int, int>, cudaGraphExec_t> graphs;
};

// Launches a phantom has taken after `steps` steps in the pack's mode; its
// ping-pong parity is their count & 1.
static int pack_launches(int64_t steps, int tblock) { return (int)(tblock == 2 ? (steps + 1) / 2 : steps); }

static int pack_layout(ceep2d_plan* const* plans, int32_t count, size_t* bytes,
                       std::vector<std::vector<std::pair<int, int>>>* cls_out,
                       std::vector<std::tuple<int, int, int>>* keys_out) {
  if (!plans || count < 1) return fail(CEEP_ERR_INVALID, "pack: no plans");
  std::vector<std::tuple<int, int, int>> keys;
  std::vector<std::vector<std::pair<int, int>>> cls;  // per class: (nsteps, plan index)
  for (int i = 0; i < count; ++i) {
    if (!plans[i]) return fail(CEEP_ERR_INVALID, "pack: null plan %d", i);
    const ceep::Fdtd2dParams& p = plans[i]->p;
    auto key = std::make_tuple(p.L, p.n_debye, p.n_lorentz);
    auto it = std::find(keys.begin(), keys.end(), key);
    if (it == keys.end()) {
      keys.push_back(key);
      cls.emplace_back();
      it = keys.end() - 1;
    }
    cls[it - keys.begin()].push_back({p.nsteps, i});
  }
  size_t b = align16(sizeof(ceep::Fdtd2dParams) * count);
  for (auto& c : cls) {
    size_t tiles = 0;
    for (auto& e : c) {
      const ceep::Fdtd2dParams& p = plans[e.second]->p;
      const int cx = ceep::fdtd2d_cells_per_block(p.L);
      tiles += (size_t)((p.nx + cx - 1) / cx) * ((p.ny + p.rows - 1) / p.rows) * p.groups;
    }
    b += align16(tiles * sizeof(ceep::PackTile));
    size_t tiles2 = 0;
    for (auto& e : c) {
      const ceep::Fdtd2dParams& p = plans[e.second]->p;
      const int cx = ceep::fdtd2d_cells_per_block(p.L) - 2;
      if (p.rows2 < 1) return fail(CEEP_ERR_INVALID, "pack: plan %d has no two-step tile height", e.second);
      tiles2 += ((size_t)((p.nx + cx - 1) / cx) * ((p.ny + p.rows2 - 1) / p.rows2) +
                 (size_t)(CEEP_PACK_FRAME_PIECES - 1) * p.nframe2) * p.groups;
    }
    b += align16(tiles2 * sizeof(ceep::PackTile));
  }
  *bytes = b;
  if (cls_out) *cls_out = cls;
  if (keys_out) *keys_out = keys;
  return CEEP_OK;
}

extern "C" int64_t ceep2d_pack_workspace_bytes(ceep2d_plan* const* plans, int32_t count) {
  size_t b = 0;
  return pack_layout(plans, count, &b, nullptr, nullptr) == CEEP_OK ? (int64_t)b : -1;
}

extern "C" int ceep2d_pack_create(ceep2d_plan* const* plans, int32_t count, void* workspace, int64_t bytes,
                                  void* stream, ceep2d_pack** out) {
  if (!out || !workspace) return fail(CEEP_ERR_INVALID, "pack: null argument");
  *out = nullptr;
  size_t need = 0;
  std::vector<std::vector<std::pair<int, int>>> cls;
  std::vector<std::tuple<int, int, int>> keys;
  int rc = pack_layout(plans, count, &need, &cls, &keys);
  if (rc != CEEP_OK) return rc;
  if ((size_t)bytes < need) return fail(CEEP_ERR_INVALID, "pack: workspace %lld < %zu bytes", (long long)bytes, need);
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  ceep2d_pack* pk = new (std::nothrow) ceep2d_pack();
  if (!pk) return fail(CEEP_ERR_INVALID, "host allocation failed");
  pk->plans.assign(plans, plans + count);
  char* ws = static_cast<char*>(workspace);
  pk->params = reinterpret_cast<ceep::Fdtd2dParams*>(ws);
  std::vector<ceep::Fdtd2dParams> hp(count);
  for (int i = 0; i < count; ++i) {
    hp[i] = plans[i]->p;
    pk->max_steps = std::max(pk->max_steps, hp[i].nsteps);
  }
  // host staging vectors must outlive the asynchronous copies: synchronise below
  std::vector<std::vector<ceep::PackTile>> host_tiles(cls.size()), host_tiles2(cls.size());
  size_t off = align16(sizeof(ceep::Fdtd2dParams) * count);
  for (size_t c = 0; c < cls.size(); ++c) {
    auto& v = cls[c];
    std::stable_sort(v.begin(), v.end(), [](const std::pair<int, int>& a, const std::pair<int, int>& b) {
      return a.first > b.first;  // longest runs first: the active tiles stay a prefix
    });
    PackClass pc;
    pc.L = std::get<0>(keys[c]);
    pc.nd = std::get<1>(keys[c]);
    pc.nl = std::get<2>(keys[c]);
    // frame test of tile (bx, by) of a gx x gy grid with frame counts fc
    auto is_frame = [](int bx, int by, int gx, int gy, const int* fc) {
      return bx < fc[0] || bx >= gx - fc[1] || by < fc[2] || by >= gy - fc[3];
    };
    std::vector<ceep::PackTile> tf, ti;
    struct End { int steps; size_t f, i; };
    std::vector<End> ends;  // per phantom: step count, frame and interior tiles so far
    for (auto& e : v) {
      const ceep::Fdtd2dParams& p = hp[e.second];
      const int cx = ceep::fdtd2d_cells_per_block(p.L);
      const int gx = (p.nx + cx - 1) / cx, gy = (p.ny + p.rows - 1) / p.rows;
      for (int g = 0; g < p.groups; ++g)
        for (int by = 0; by < gy; ++by)
          for (int bx = 0; bx < gx; ++bx)
            (is_frame(bx, by, gx, gy, p.frame1) ? tf : ti).push_back({e.second, bx * cx, by * p.rows, g, p.rows});
      ends.push_back({p.nsteps, tf.size(), ti.size()});
    }
    pc.nf = (int)tf.size();
    std::vector<ceep::PackTile>& tl = host_tiles[c];
    tl = tf;
    tl.insert(tl.end(), ti.begin(), ti.end());
    pc.act_f.assign(pk->max_steps, 0);
    pc.act_i.assign(pk->max_steps, 0);
    for (int t = 0; t < pk->max_steps; ++t)
      for (auto& en : ends)
        if (en.steps > t) {
          pc.act_f[t] = (int)en.f;
          pc.act_i[t] = (int)en.i;
        }
    pc.tiles = reinterpret_cast<ceep::PackTile*>(ws + off);
    off += align16(tl.size() * sizeof(ceep::PackTile));
    // the two-step tables (same phantom order)
    std::vector<ceep::PackTile> t2f, t2i;
    std::vector<End> ends2;
    for (auto& e : v) {
      const ceep::Fdtd2dParams& p = hp[e.second];
      const int cx = ceep::fdtd2d_cells_per_block(p.L) - 2;
      const int gx = (p.nx + cx - 1) / cx, gy = (p.ny + p.rows2 - 1) / p.rows2;
      for (int g = 0; g < p.groups; ++g)
        for (int by = 0; by < gy; ++by)
          for (int bx = 0; bx < gx; ++bx)
            if (is_frame(bx, by, gx, gy, p.frame2)) {  // frame tiles as row pieces
              const int fp = CEEP_PACK_FRAME_PIECES;
              for (int k = 0; k < fp; ++k)
                t2f.push_back({e.second, bx * cx - 1, by * p.rows2 + k * p.rows2 / fp, g,
                               (k + 1) * p.rows2 / fp - k * p.rows2 / fp});
            } else {
              t2i.push_back({e.second, bx * cx - 1, by * p.rows2, g, p.rows2});
            }
      ends2.push_back({p.nsteps, t2f.size(), t2i.size()});
    }
    pc.nf2 = (int)t2f.size();
    std::vector<ceep::PackTile>& t2 = host_tiles2[c];
    t2 = t2f;
    t2.insert(t2.end(), t2i.begin(), t2i.end());
    const int pairs = (pk->max_steps + 1) / 2;
    for (auto* vec : {&pc.act2_f, &pc.act2_i, &pc.tail_f_lo, &pc.tail_f_hi, &pc.tail_i_lo, &pc.tail_i_hi})
      vec->assign(pairs, 0);
    for (int t = 0; t < pairs; ++t) {
      for (size_t k = 0; k < ends2.size(); ++k) {
        if (ends2[k].steps >= 2 * t + 2) {
          pc.act2_f[t] = (int)ends2[k].f;
          pc.act2_i[t] = (int)ends2[k].i;
          pc.tail_f_lo[t] = (int)ends[k].f;
          pc.tail_i_lo[t] = (int)ends[k].i;
        }
        if (ends2[k].steps >= 2 * t + 1) {
          pc.tail_f_hi[t] = (int)ends[k].f;
          pc.tail_i_hi[t] = (int)ends[k].i;
        }
      }
    }
    pc.tiles2 = reinterpret_cast<ceep::PackTile*>(ws + off);
    off += align16(t2.size() * sizeof(ceep::PackTile));
    pk->classes.push_back(pc);
  }
  cudaError_t e = cudaMemcpyAsync(pk->params, hp.data(), sizeof(ceep::Fdtd2dParams) * count,
                                  cudaMemcpyHostToDevice, s);
  for (size_t c = 0; c < cls.size() && e == cudaSuccess; ++c) {
    e = cudaMemcpyAsync(pk->classes[c].tiles, host_tiles[c].data(), host_tiles[c].size() * sizeof(ceep::PackTile),
                        cudaMemcpyHostToDevice, s);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(pk->classes[c].tiles2, host_tiles2[c].data(),
                          host_tiles2[c].size() * sizeof(ceep::PackTile), cudaMemcpyHostToDevice, s);
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) {
    delete pk;
    return ceep::cuda_fail(e, "pack: table upload");
  }
  for (auto* pl : pk->plans) pl->cur = 0;
  *out = pk;
  return CEEP_OK;
}

// Launch steps [step0, step0 + nsteps) of the classes [c0, c1) on stream s.
static int pack_steps(ceep2d_pack* pk, int64_t step0, int64_t nsteps, cudaStream_t s, size_t c0, size_t c1) {
  if (pk->tblock == 2) {
    // pairs of steps: par is the pair index & 1 for every phantom still running
    for (int64_t t = step0 / 2; 2 * t < step0 + nsteps; ++t)
      for (size_t ci = c0; ci < c1; ++ci) {
        auto& c = pk->classes[ci];
        cudaError_t e = ceep::fdtd2d_launch_packed(c.L, c.nd, c.nl, c.tiles2, c.act2_f[t], c.tiles2 + c.nf2,
                                                   c.act2_i[t], pk->params, (int)(2 * t), (int)(t & 1), true, s);
        if (e == cudaSuccess)
          e = ceep::fdtd2d_launch_packed(c.L, c.nd, c.nl, c.tiles + c.tail_f_lo[t], c.tail_f_hi[t] - c.tail_f_lo[t],
                                         c.tiles + c.nf + c.tail_i_lo[t], c.tail_i_hi[t] - c.tail_i_lo[t],
                                         pk->params, (int)(2 * t), (int)(t & 1), false, s);
        if (e != cudaSuccess) return ceep::cuda_fail(e, "packed step launch");
      }
    return CEEP_OK;
  }
  for (int64_t t = step0; t < step0 + nsteps; ++t)
    for (size_t ci = c0; ci < c1; ++ci) {
      auto& c = pk->classes[ci];
      cudaError_t e = ceep::fdtd2d_launch_packed(c.L, c.nd, c.nl, c.tiles, c.act_f[t], c.tiles + c.nf, c.act_i[t],
                                                 pk->params, (int)t, (int)(t & 1), false, s);
      if (e != cudaSuccess) return ceep::cuda_fail(e, "packed step launch");
    }
  return CEEP_OK;
}

// All classes: interleaved on s, or (concurrent packing) class 0 on s and
// class c on side stream c-1, forked from and joined back to s.
static int pack_all(ceep2d_pack* pk, int64_t step0, int64_t nsteps, cudaStream_t s) {
  const size_t nc = pk->classes.size();
  if (!pk->concurrent || nc < 2) return pack_steps(pk, step0, nsteps, s, 0, nc);
  cudaError_t e = cudaEventRecord(pk->events[0], s);
  for (size_t c = 1; c < nc && e == cudaSuccess; ++c) e = cudaStreamWaitEvent(pk->side[c - 1], pk->events[0], 0);
  if (e != cudaSuccess) return ceep::cuda_fail(e, "pack: fork");
  int rc = pack_steps(pk, step0, nsteps, s, 0, 1);
  for (size_t c = 1; c < nc; ++c) {
    const int r = pack_steps(pk, step0, nsteps, pk->side[c - 1], c, c + 1);
    if (rc == CEEP_OK) rc = r;
    e = cudaEventRecord(pk->events[c], pk->side[c - 1]);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s, pk->events[c], 0);
    if (e != cudaSuccess && rc == CEEP_OK) rc = ceep::cuda_fail(e, "pack: join");
  }
  return rc;
}

extern "C" int ceep2d_pack_set_packing(ceep2d_pack* pk, int concurrent) {
  if (!pk || (concurrent != 0 && concurrent != 1))
    return fail(CEEP_ERR_INVALID, "pack: packing %d (0 or 1)", concurrent);
  if (concurrent && pk->side.empty() && pk->classes.size() > 1) {
    const size_t nc = pk->classes.size();
    cudaError_t e = cudaSuccess;
    for (size_t c = 0; c < nc && e == cudaSuccess; ++c) {
      cudaEvent_t ev;
      e = cudaEventCreateWithFlags(&ev, cudaEventDisableTiming);
      if (e == cudaSuccess) pk->events.push_back(ev);
    }
    for (size_t c = 1; c < nc && e == cudaSuccess; ++c) {
      cudaStream_t st;
      e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
      if (e == cudaSuccess) pk->side.push_back(st);
    }
    if (e != cudaSuccess) return ceep::cuda_fail(e, "pack: side streams");
  }
  pk->concurrent = concurrent;
  return CEEP_OK;
}

extern "C" int ceep2d_pack_packing(const ceep2d_pack* pk) { return pk ? pk->concurrent : -1; }

extern "C" int ceep2d_pack_set_temporal_block(ceep2d_pack* pk, int steps) {
  if (!pk || (steps != 1 && steps != 2)) return fail(CEEP_ERR_INVALID, "pack: temporal block %d (1 or 2)", steps);
  pk->tblock = steps;
  return CEEP_OK;
}

extern "C" int ceep2d_pack_temporal_block(const ceep2d_pack* pk) { return pk ? pk->tblock : 0; }

extern "C" int ceep2d_pack_run(ceep2d_pack* pk, int64_t step0, int64_t nsteps, void* stream, int use_graph) {
  if (!pk) return fail(CEEP_ERR_INVALID, "null pack");
  if (step0 < 0 || nsteps < 0 || step0 + nsteps > pk->max_steps)
    return fail(CEEP_ERR_INVALID, "pack: steps [%lld, %lld) outside [0, %d)", (long long)step0,
                (long long)(step0 + nsteps), pk->max_steps);
  if (pk->tblock == 2 && (step0 % 2 || ((step0 + nsteps) % 2 && step0 + nsteps != pk->max_steps)))
    return fail(CEEP_ERR_INVALID, "pack: two steps per launch need even step bounds (or the last step)");
  for (auto* pl : pk->plans)
    if (pl->cur != (pack_launches(std::min<int64_t>(step0, pl->p.nsteps), pk->tblock) & 1))
      return fail(CEEP_ERR_INVALID, "pack: a plan's state is not at step %lld", (long long)step0);
  if (nsteps == 0) return CEEP_OK;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  int rc = CEEP_OK;
  if (!use_graph || s == nullptr) {
    rc = pack_all(pk, step0, nsteps, s);
  } else {
    auto key = std::make_tuple(step0, nsteps, pk->tblock, pk->concurrent);
    auto it = pk->graphs.find(key);
    if (it == pk->graphs.end()) {
      cudaGraph_t g;
      cudaError_t e = cudaStreamBeginCapture(s, cudaStreamCaptureModeThreadLocal);
      if (e != cudaSuccess) return ceep::cuda_fail(e, "cudaStreamBeginCapture");
      rc = pack_all(pk, step0, nsteps, s);
      e = cudaStreamEndCapture(s, &g);
      if (rc != CEEP_OK) { if (e == cudaSuccess) cudaGraphDestroy(g); return rc; }
      if (e != cudaSuccess) return ceep::cuda_fail(e, "cudaStreamEndCapture");
      cudaGraphExec_t ex;
      e = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (e != cudaSuccess) return ceep::cuda_fail(e, "cudaGraphInstantiate");
      it = pk->graphs.emplace(key, ex).first;
    }
    cudaError_t e = cudaGraphLaunch(it->second, s);
    if (e != cudaSuccess) return ceep::cuda_fail(e, "cudaGraphLaunch");
  }
  if (rc == CEEP_OK)
    for (auto* pl : pk->plans) pl->cur = pack_launches(std::min<int64_t>(step0 + nsteps, pl->p.nsteps), pk->tblock) & 1;
  return rc;
}

extern "C" int ceep2d_pack_tiles(const ceep2d_pack* pk, int32_t step) {
  if (!pk || step < 0 || step >= pk->max_steps) return -1;
  int n = 0;
  for (auto& c : pk->classes) n += c.act_f[step] + c.act_i[step];
  return n;
}

extern "C" int ceep2d_pack_destroy(ceep2d_pack* pk) {
  if (!pk) return CEEP_OK;
  for (auto& kv : pk->graphs) cudaGraphExecDestroy(kv.second);
  for (auto st : pk->side) cudaStreamDestroy(st);
  for (auto ev : pk->events) cudaEventDestroy(ev);
  delete pk;
  return CEEP_OK;
}

/*
 * ceep_b200 — C ABI of the B200-native batched multistatic FDTD path.
 *
 * Drop-in boundary for the hot path of the reference project
 * (shahzaibshazoo/ceep-v1).  The reference has no FFI: its seam is the Python
 * solver classes plus the global array-module switch.  Each entry point below
 * replaces one piece of that path; the reference location is cited beside it.
 *
 * Conventions
 *   - Every buffer argument is a DEVICE pointer owned by the caller (in the
 *     Python host code: torch tensors).  The library never allocates device
 *     memory, never calls exit/abort, and never synchronises the device
 *     except where a function says so.
 *   - Field layout is (y, x, tx) in 2D and (z, y, x, tx) in 3D, tx innermost,
 *     tx padded to `ntx_pad` (a multiple of 4; a multiple of 32 above 32).
 *   - Functions return 0 on success or a ceep_status code; the message of
 *     the last failure on the calling thread is returned by ceep_last_error().
 *   - `stream` is a cudaStream_t (NULL = legacy default stream).
 *   - A plan is not thread-safe; use one plan per host thread.
 */
#ifndef CEEP_B200_H
#define CEEP_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef enum ceep_status {
  CEEP_OK = 0,
  CEEP_ERR_INVALID = 1,     /* bad argument (sizes, positions, null pointer) */
  CEEP_ERR_CUDA = 2,        /* a CUDA runtime call failed                    */
  CEEP_ERR_UNSUPPORTED = 3, /* configuration outside what is compiled in     */
  CEEP_ERR_TIMEOUT = 4,     /* a bounded device wait gave up                 */
  CEEP_ERR_NONFINITE = 5    /* NaN/Inf found by the sentinel                 */
} ceep_status;

/* Library version and last error (thread-local message). */
int ceep_version(void);
const char* ceep_last_error(void);

/* ------------------------------------------------------------------------
 * 2D TMz batched FDTD.
 * Replaces BatchedFDTD2D.run()'s time loop, src/ceep/solvers/fdtd_2d_batched.py:454-526
 * (interior H :471-483, _apply_h_cpml :272-334, interior E :491-498,
 *  _apply_e_cpml :336-406, edge zeroing :503-507, source :509-515,
 *  probes :517-526), with the Debye/Lorentz ADE of
 *  src/ceep/materials/dispersive.py:364-404 composed into the interior E update.
 * ---------------------------------------------------------------------- */
typedef struct ceep2d_desc {
  int32_t nx, ny;          /* grid (x, y)                                    */
  int32_t cpml;            /* CPML thickness n (0, or 2 <= n)                */
  int32_t ntx, ntx_pad;    /* transmit events and padded lane count          */
  int32_t nprobe;          /* receivers                                      */
  int32_t nsteps;          /* length of waveform and of each probe series    */
  int32_t n_debye, n_lorentz; /* ADE poles per cell (0..2 each)              */
  float db;                /* dt / mu0                                       */
  float inv_dx;            /* 1 / dx (dx == dy)                              */
  float dt;                /* time step (ADE dE/dt)                          */
  /* Per-TX arrays are split into groups of at most 32 transmit events:
   * G = ntx_pad / min(ntx_pad, 32) groups, each group's array contiguous, so
   * a field is (G, ny, nx, ntx_pad / G) floats (for ntx_pad <= 32 simply
   * (ny, nx, ntx_pad)).
   * ping-pong state, each (G, ny, nx, ntx_pad/G) float; [k] = buffer k      */
  float* ez[2];
  float* hx[2];
  float* hy[2];
  /* H-CPML psi, ping-pong: x strips (G, ny, 2n, .), y strips (G, 2n, nx, .) */
  float* psi_hy[2];
  float* psi_hx[2];
  /* E-CPML psi, ping-pong, same shapes as above                             */
  float* psi_ezx[2];
  float* psi_ezy[2];
  /* ADE currents, ping-pong: (G, poles, ny, nx, .); Lorentz keeps J^{n-1}   */
  float* j[2];             /* n_debye + n_lorentz planes                     */
  float* j_prev[2];        /* n_lorentz planes                               */
  const float* coef;       /* (ny, nx, 4): ca, cb, dt/(eps_r eps0), 0        */
  const float* ade_coef;   /* (poles, ny, nx, 4): Debye k1,k2,gamma ; Lorentz k1,k2,k3 */
  const float* cpml_b;     /* (n)                                            */
  const float* cpml_c;     /* (n)                                            */
  const int32_t* src_xy;   /* (ntx, 2) source cell per transmit event        */
  const int32_t* prb_xy;   /* (nprobe, 2)                                    */
  const uint8_t* row_flags;/* (ny): bit0 a source on this row, bit1 a probe  */
  const float* waveform;   /* (nsteps)                                       */
  float* probes;           /* (ntx, nprobe, nsteps) output series            */
  int32_t* status;         /* device word, 0 = ok; a bounded wait that gives
                              up writes CEEP_ERR_TIMEOUT (may be NULL)        */
  int32_t rows_per_block;  /* 0 = chosen to fill whole waves of the GPU     */
} ceep2d_desc;

typedef struct ceep2d_plan ceep2d_plan;

/* Validate the descriptor and build a plan (host memory only). */
int ceep2d_plan_create(const ceep2d_desc* desc, ceep2d_plan** out);
/* Advance `nsteps` steps starting at global step `step0`.  use_graph != 0
 * captures the launches once per (step0, nsteps) and replays the CUDA graph on
 * later calls.  Every launch (one or two steps) reads the current ping-pong
 * buffer and writes the other one. */
int ceep2d_plan_run(ceep2d_plan* plan, int64_t step0, int64_t nsteps, void* stream, int use_graph);
int ceep2d_plan_destroy(ceep2d_plan* plan);
/* Number of kernel launches one step issues with a temporal block of 1. */
int ceep2d_launches_per_step(const ceep2d_plan* plan);
/* Steps per launch: 1 (one fused step per launch), or 2 (temporal block of
 * two: each state word is read once and written once per two steps; the
 * same arithmetic, bit-identical results).  No counterpart in the reference.
 * A new plan uses 1; the Python solver sets 2. */
int ceep2d_plan_set_temporal_block(ceep2d_plan* plan, int steps);
int ceep2d_plan_temporal_block(const ceep2d_plan* plan);
/* Two-step launches as two kernels (1): the frame tiles (CPML strips, grid
 * edges) on a high-priority stream of the plan beside a kernel of the
 * interior tiles, which without the strip code and psi slices fits four
 * blocks per SM; 0 (the default): one kernel for every tile.  Same
 * arithmetic, bit-identical results.  No counterpart in the reference. */
int ceep2d_plan_set_frame_split(ceep2d_plan* plan, int32_t on);
/* Kernel launches a ceep2d_plan_run of `nsteps` steps issues (step kernels
 * only; the NaN/Inf sentinel's scans are not counted). */
int64_t ceep2d_plan_launches(const ceep2d_plan* plan, int64_t nsteps);
/* NaN/Inf sentinel.  Replaces the reference's after-the-fact check
 * `np.all(np.isfinite(signal))` (tests/test_fdtd_3d_batched.py:240-244)
 * with a device scan: when the plan has a status word, a small kernel scans
 * the current Ez and the probe samples recorded since its last scan, after
 * every `interval` steps and after the last step of every run range
 * (interval 0, the default: only the latter), and records
 * CEEP_ERR_NONFINITE in the status word on a NaN or Inf. */
int ceep2d_plan_set_sentinel(ceep2d_plan* plan, int32_t interval);
/* Bound of every mbarrier wait of the step kernels, in ns (default 1 s).  A
 * wait that runs out records CEEP_ERR_TIMEOUT in the status word and the
 * block leaves after its copies in flight have landed (no counterpart in
 * the reference, whose CuPy kernels have no device waits). */
int ceep2d_plan_set_wait_limit(ceep2d_plan* plan, uint64_t ns);
/* Failure injection for tests of the bounded waits (no counterpart in the
 * reference): the producer of every block issues no copies for grid row
 * `row`, so the consumers' waits on that row run out after the wait limit
 * and the launch reports CEEP_ERR_TIMEOUT.  The state it leaves is not a
 * valid simulation state.  -1 (the default) turns it off. */
int ceep2d_plan_inject_copy_fault(ceep2d_plan* plan, int32_t row);
/* Which ping-pong buffer (0 or 1) holds the current state; reset sets it to 0
 * (the caller zeroes the state buffers). */
int ceep2d_plan_current_buffer(const ceep2d_plan* plan);
int ceep2d_plan_reset(ceep2d_plan* plan);
/* sizeof(ceep2d_desc), for binding layers to check their struct mirror. */
int64_t ceep2d_desc_size(void);
/* Rows per block the plan launches with (chosen at creation when 0). */
int ceep2d_plan_rows(const ceep2d_plan* plan);
/* As ceep2d_plan_run, and also store Ez^{n+1} (and J^{n+1} when save_j is
 * given) of every step n into slot n + 1 - save_base of save_ez
 * (slots, G, ny, nx, .) / save_j (slots, G, poles, ny, nx, .): the forward
 * values the adjoint needs (J only for tau gradients).  J entries outside
 * the interior E region are never written (the caller zeroes the buffer
 * once). */
int ceep2d_plan_run_save(ceep2d_plan* plan, int64_t step0, int64_t nsteps, void* stream, int use_graph,
                         float* save_ez, float* save_j, int64_t save_base);
/* Select which ping-pong buffer holds the current state (after the caller
 * restores a checkpoint into it). */
int ceep2d_plan_set_current_buffer(ceep2d_plan* plan, int cur);

/* ------------------------------------------------------------------------
 * Packed launch of many 2D plans (phantoms of uneven size, step count, TX
 * count and ADE model).  No counterpart in the reference, which runs one
 * BatchedFDTD2D per phantom (scripts/generate_corrected_dataset.py:139-149).
 * Each time step is one launch per (lane width, ADE shape) class covering the
 * tiles of every plan of that class still running; plans are ordered by
 * decreasing step count so the running tiles form a prefix of the class's
 * tile table.  Per-plan parameters and tile tables live in the caller's
 * workspace (ceep2d_pack_workspace_bytes); every plan must be at step 0
 * (freshly created or reset) when the pack is created.
 * ---------------------------------------------------------------------- */
typedef struct ceep2d_pack ceep2d_pack;
int64_t ceep2d_pack_workspace_bytes(ceep2d_plan* const* plans, int32_t count);
int ceep2d_pack_create(ceep2d_plan* const* plans, int32_t count, void* workspace, int64_t bytes,
                       void* stream, ceep2d_pack** out);
/* Steps [step0, step0 + nsteps) of the longest plan; shorter plans stop at
 * their own step count.  use_graph != 0 captures and replays a CUDA graph. */
int ceep2d_pack_run(ceep2d_pack* pack, int64_t step0, int64_t nsteps, void* stream, int use_graph);
/* Number of tiles (blocks) launched at `step`, over all classes. */
int ceep2d_pack_tiles(const ceep2d_pack* pack, int32_t step);
/* Steps per launch, 1 or 2 (default 1).  With 2 every launch advances each
 * running plan two steps with the temporal-block kernel (its own tile
 * table: tile height = each plan's two-step rows); a plan with an odd step
 * count takes its last step alone.  Runs then start at an even step and end
 * at an even step or the last one.  Set before the first run. */
int ceep2d_pack_set_temporal_block(ceep2d_pack* pack, int steps);
int ceep2d_pack_temporal_block(const ceep2d_pack* pack);
/* Packing of the classes (lane width x ADE shape) in time, an autotuner
 * choice with no counterpart in the reference (whose dataset generator runs
 * one solver per phantom, scripts/generate_corrected_dataset.py:139-149):
 * 0 (default) launches every class's step on the caller's stream in turn;
 * 1 gives each class beyond the first its own stream (created here, owned by
 * the pack), so the classes' launch chains, which touch disjoint phantoms,
 * run side by side, forked from and joined back to the caller's stream. */
int ceep2d_pack_set_packing(ceep2d_pack* pack, int concurrent);
int ceep2d_pack_packing(const ceep2d_pack* pack);
int ceep2d_pack_destroy(ceep2d_pack* pack);

/* ------------------------------------------------------------------------
 * Adjoint (reverse-mode) of the 2D step: no counterpart in the reference
 * (src/ceep/ai/__init__.py only announces a differentiable solver).  It is
 * the exact transpose of the fused step above, run backwards in time; per
 * cell it accumulates (over transmit events and steps) the gradients of the
 * loss with respect to ca, cb, the Debye k1, k2, gamma of each Debye pole
 * and the k2 of each Lorentz pole (the transposed two-level Lorentz
 * recurrence of dispersive.py:278-299 / :396-404).  One launch per step.
 * Every adjoint state array is a ping-pong pair shaped like the forward's
 * (both halves zeroed by the caller before the first run).
 * ---------------------------------------------------------------------- */
typedef struct ceep2d_adjoint_desc {
  float* ez[2];            /* adjoint Ez, (G, ny, nx, .)                     */
  float* hx[2];            /* adjoint Hx / Hy                                */
  float* hy[2];
  float* psi_hx[2];        /* adjoint H-CPML psi (forward shapes)            */
  float* psi_hy[2];
  float* psi_ezx[2];       /* adjoint E-CPML psi                             */
  float* psi_ezy[2];
  float* j[2];             /* adjoint currents of every pole (Debye first,
                              then Lorentz; the forward J's shape)           */
  float* jp[2];            /* adjoint Lorentz J_prev (the forward j_prev's
                              shape); may be NULL without Lorentz poles      */
  double* grad;            /* (G, ny, nx, KP), KP = 2 + 3*poles rounded up to
                              even: per TX group and cell d/dca, d/dcb, then
                              per Debye pole d/dk1, d/dk2, d/dgamma and per
                              Lorentz pole d/dk1, d/dk2, d/dk3 (only d/dk2 is
                              formed for Lorentz poles: k1 and k3 depend on
                              omega_0 and delta alone), then a zero pad;
                              accumulated                                    */
  const float* probe_grad; /* (ntx, nprobe, nsteps) dLoss/dprobe             */
  int32_t grad_tau;        /* nonzero: also d/dk1 and d/dgamma, which depend
                              on tau only and need the forward's saved J;
                              0: those slots stay 0 and ceep2d_adjoint_run
                              takes seg_j = NULL                             */
} ceep2d_adjoint_desc;

typedef struct ceep2d_adjoint ceep2d_adjoint;
int ceep2d_adjoint_create(const ceep2d_plan* plan, const ceep2d_adjoint_desc* desc, ceep2d_adjoint** out);
/* Transposed steps n = step_hi-1 down to step_hi-nsteps.  Forward values come
 * from a segment saved by ceep2d_plan_run_save: Ez^n is slot n - seg_base of
 * seg_ez (slot 0 = the segment's starting state), J^n likewise. */
int ceep2d_adjoint_run(ceep2d_adjoint* adj, int64_t step_hi, int64_t nsteps, const float* seg_ez,
                       const float* seg_j, int64_t seg_base, void* stream);
int ceep2d_adjoint_reset(ceep2d_adjoint* adj);
int ceep2d_adjoint_destroy(ceep2d_adjoint* adj);
int64_t ceep2d_adjoint_desc_size(void);
/* Rows of the segment one block of the adjoint walks per step. */
int ceep2d_adjoint_rows(const ceep2d_adjoint* adj);
/* Tile height (rows per block) of the adjoint launch, 0 for the automatic
 * choice (no reference counterpart: a launch-geometry setting). */
int ceep2d_adjoint_set_rows(ceep2d_adjoint* adj, int32_t rows);

/* ------------------------------------------------------------------------
 * 3D batched Yee FDTD.
 * Replaces BatchedFDTD3D.run()'s time loop, src/ceep/solvers/fdtd_3d_batched.py:918-958
 * (_update_h_fields :753-818, _apply_h_cpml_x/y/z :398-586,
 *  _update_e_fields :820-884, low-face zeroing :936-944, source :949-951,
 *  probes :956-958), with optional Debye/Lorentz currents on each E component.
 * Per step: the H half-step as two launches over disjoint cells (the box
 * inside every interior box and off every CPML face, and the shell around it
 * on a side stream of the plan), the E half-step, and the source/probe
 * epilogue; all state is updated in place.
 * ---------------------------------------------------------------------- */
typedef struct ceep3d_desc {
  int32_t nx, ny, nz;
  int32_t cpml;
  int32_t ntx, ntx_pad, nprobe, nsteps;
  int32_t n_debye, n_lorentz;
  float inv_dx, dt;
  /* fields, each (G, nz, ny, nx, ntx_pad/G) float, G = TX groups of <= 32 */
  float *ex, *ey, *ez, *hx, *hy, *hz;
  /* CPML psi: x faces (G, nz, ny, 2n, .), y faces (G, nz, 2n, nx, .),
   * z faces (G, 2n, ny, nx, .); psi_hxy/psi_hzy act on Hy/Hz, psi_hyx/psi_hzx
   * on Hx/Hz, psi_hxz/psi_hyz on Hx/Hy                                        */
  float *psi_hxy, *psi_hzy, *psi_hyx, *psi_hzx, *psi_hxz, *psi_hyz;
  float* j;                /* (G, poles, 3, nz, ny, nx, .)                   */
  float* j_prev;           /* (G, n_lorentz, 3, nz, ny, nx, .)               */
  const float* coef;       /* (nz, ny, nx, 4): da, db, ca, cb                */
  const float* ade_coef;   /* (poles, nz, ny, nx, 4)                         */
  const float* cpml_b;
  const float* cpml_c;
  const int32_t* src_xyz;  /* (ntx, 3) */
  const int32_t* prb_xyz;  /* (nprobe, 3) */
  const float* waveform;   /* (nsteps) */
  float* probes;           /* (ntx, nprobe, nsteps) */
  int32_t z_rows;          /* z segment per thread, 0 = default              */
  int32_t shell_z_rows;    /* z walk of the H shell launch, 0 = default      */
} ceep3d_desc;

typedef struct ceep3d_plan ceep3d_plan;
int ceep3d_plan_create(const ceep3d_desc* desc, ceep3d_plan** out);
int ceep3d_plan_run(ceep3d_plan* plan, int64_t step0, int64_t nsteps, void* stream, int use_graph);
/* As ceep3d_plan_run, and also store the three E components of every step n,
 * as the E half-step leaves them (before the source), into slot
 * n + 1 - save_base of save_e, a (slots, 3, G, nzi, nyi, nxi, .) float array
 * over the interior E box [n+1, N-n)^3 (nxi = nx - 2n - 1 and so on), the
 * only cells the E half-step updates.  With interior_only the H half-step
 * skips the CPML shell (H outside [n, N-n)^3 and the psi arrays stay as they
 * were): E, the H box, the currents and the probes come out bit-identical,
 * since nothing in the shell reaches them, for a fraction of the traffic. */
int ceep3d_plan_run_save(ceep3d_plan* plan, int64_t step0, int64_t nsteps, void* stream, int use_graph,
                         float* save_e, int64_t save_base, int interior_only);
int ceep3d_plan_destroy(ceep3d_plan* plan);
int64_t ceep3d_desc_size(void);

/* ------------------------------------------------------------------------
 * Non-batched 2D FDTD, TMz or TEz, one field set.
 * Replaces FDTD2D.step()/run() (src/ceep/solvers/fdtd_2d.py:111-260 through
 * src/ceep/solvers/fdtd_base.py:158-210) with the boundaries PEC
 * (src/ceep/boundaries/absorbing.py:48-78), MurABC (:80-172, last in the
 * list only) and CFS-CPML (:174-561, one per plan), soft sources and the
 * probe / monitor recording of FDTD2D._record (fdtd_2d.py:277-291).
 * Fields are (nx, ny) float with y fastest (the reference's arrays).
 * ---------------------------------------------------------------------- */
typedef struct ceep2s_desc {
  int32_t nx, ny;
  int32_t mode;             /* 0 TMz: f0 Ez, f1 Hx, f2 Hy; 1 TEz: f0 Hz, f1 Ex, f2 Ey */
  int32_t nsteps;
  float inv_dx, inv_dy;
  float dt_mu0, dt_eps0;    /* scale of the CPML H and E corrections          */
  float mur_kx, mur_ky;     /* (c dt - d) / (c dt + d)                         */
  float *f0[2], *f1[2], *f2[2];  /* ping-pong: the plan's current half holds
                               the state (starts at 0)                         */
  const float* coef_e;      /* (nx, ny, 2): ca, cb                             */
  const float* coef_h;      /* (nx, ny, 2): da, db                             */
  int32_t n_ops;            /* boundary operations in list order (<= 4):      */
  int32_t ops[4];           /* 1 CPML, 2 PEC, 3 Mur (Mur last)                 */
  int32_t cpml_t;           /* CPML thickness                                  */
  const float* cpml;        /* (8, t): be_x ce_x bh_x ch_x be_y ce_y bh_y ch_y */
  float* psi_e;             /* E psi: x-lo, x-hi (t, ny) each, then y-lo, y-hi
                               (nx, t) each; zeroed by the caller              */
  float* psi_h[2];          /* H psi, same layout, ping-pong like the fields   */
  float* mur_prev;          /* 2 x (2 ny + 2 nx), zeroed by the caller         */
  int32_t nsrc;
  int32_t hz_sources;       /* nonzero: TEz sources on Hz (field 0) exist      */
  const int32_t* src;       /* (nsrc, 3) x, y, field; stable-sorted by x       */
  const int32_t* src_row;   /* (nx + 1) offsets of each x in src               */
  const float* waveform;    /* (nsrc, nsteps) in the order of src              */
  int32_t nrec;
  const int32_t* rec;       /* (nrec, 2) flat cell index, field                */
  float* rec_out;           /* (nrec, nsteps)                                  */
  int32_t snap_field, snap_interval;
  float* snapshots;         /* (ceil(nsteps / interval), nx, ny) or NULL       */
} ceep2s_desc;

typedef struct ceep2s_plan ceep2s_plan;
int ceep2s_plan_create(const ceep2s_desc* desc, ceep2s_plan** out);
/* Steps step0 .. step0+nsteps-1 (the step index selects the waveform column,
 * the record column and the Mur state half).  With use_graph and a stream, a
 * range is captured into a CUDA graph the second time it is asked for and
 * replayed from then on; its first run launches directly, so a one-off run
 * pays no capture. */
int ceep2s_plan_run(ceep2s_plan* plan, int64_t step0, int64_t nsteps, void* stream, int use_graph);
/* The half (0 or 1) of the ping-pong arrays that holds the current state;
 * each step flips it. */
int ceep2s_plan_current_buffer(const ceep2s_plan* plan);
int ceep2s_plan_set_current_buffer(ceep2s_plan* plan, int cur);
int ceep2s_plan_destroy(ceep2s_plan* plan);
int64_t ceep2s_desc_size(void);

/* ------------------------------------------------------------------------
 * 3D adjoint: the exact transpose of the 3D step restricted to what the
 * probe series depends on (the E interior [n+1, N-n)^3 and the H box
 * [n, N-n)^3, which no CPML face touches), giving per-cell gradients of a
 * loss of the probe series with respect to ca, cb and each Debye k2.  No
 * reference counterpart (the reference's 3D solver has no gradient); the
 * forward it transposes is fdtd_3d_batched.py:886-985.
 * State arrays (caller-owned, zeroed before the first run):
 *   mu, nu: (3, G, nz, ny, nx, .) float;  lj: the forward J layout;
 *   grad:   (G, 2 + poles, nz-2n-1, ny-2n-1, nx-2n-1) double, per interior
 *           cell ca, cb, then k2 of each Debye pole, summed over steps/TX.
 * ---------------------------------------------------------------------- */
typedef struct ceep3d_adjoint_desc {
  float* mu;                /* adjoint E plus (k2/dt) adjoint J               */
  float* nu;                /* adjoint H (before the next step's da)          */
  float* lj;                /* adjoint Debye currents                         */
  double* grad;
  const float* probe_grad;  /* (ntx, nprobe, nsteps) dLoss/dprobe             */
} ceep3d_adjoint_desc;

typedef struct ceep3d_adjoint ceep3d_adjoint;
int ceep3d_adjoint_create(const ceep3d_plan* plan, const ceep3d_adjoint_desc* desc, ceep3d_adjoint** out);
/* Adjoint steps step_hi-1 down to step_hi-nsteps; seg_e holds the slots that
 * ceep3d_plan_run_save wrote with save_base = seg_base, slot 0 being a copy of
 * the interior E box at step seg_base (source included). */
int ceep3d_adjoint_run(ceep3d_adjoint* adj, int64_t step_hi, int64_t nsteps, const float* seg_e,
                       int64_t seg_base, void* stream);
int32_t ceep3d_adjoint_grad_slots(const ceep3d_adjoint* adj);
int ceep3d_adjoint_destroy(ceep3d_adjoint* adj);
int64_t ceep3d_adjoint_desc_size(void);

/* ------------------------------------------------------------------------
 * On-device DFT of the probe series into the S-matrix.
 * Replaces the DFTMonitor accumulation of src/ceep/solvers/dft.py:55-90 run
 * over every (tx, rx) series, laid out as MultistaticSParameters.s_matrix
 * (src/ceep/solvers/s_params.py:77-79): out[f, rx, tx] (complex64).
 *   series  : (ntx, nprobe, nsteps) float
 *   twiddle : (nfreq, nsteps) float2 = (cos(w n dt) dt, -sin(w n dt) dt),
 *             built in FP64 on the host and rounded once
 *   s_out   : (nfreq, nprobe, ntx) float2
 * ---------------------------------------------------------------------- */
int ceep_dft(const float* series, const float* twiddle, float* s_out,
             int32_t ntx, int32_t nprobe, int32_t nsteps, int32_t nfreq, void* stream);

/* ------------------------------------------------------------------------
 * Frequency-domain delay-and-sum image.
 * Replaces DelayAndSumBeamformer._reconstruct_das,
 * src/ceep/imaging/beamforming.py:210-257 (delays :146-182, pixel positions
 * :73-83, velocity :144).
 *   s       : (nfreq, nant, nant) float2, s[f, rx, tx] (frequency-masked)
 *   kfreq   : (nfreq) float, 2*pi*f / v
 *   ant_xy  : (nant, 2) float, antenna positions in metres
 *   px0,py0 : position of pixel (0,0) in metres; pix = pixel pitch
 *   work    : caller scratch, ceep_das_workspace_bytes() bytes
 *   image   : (nx_pix, ny_pix) float, |sum|, normalised to (I-min)/max when
 *             normalize != 0
 * ---------------------------------------------------------------------- */
int64_t ceep_das_workspace_bytes(int32_t nx_pix, int32_t ny_pix, int32_t nfreq);
int ceep_das(const float* s, const float* kfreq, const float* ant_xy,
             int32_t nfreq, int32_t nant, int32_t nx_pix, int32_t ny_pix,
             float px0, float py0, float pix, int normalize,
             void* work, float* image, void* stream);

/* ------------------------------------------------------------------------
 * Frequency-domain delay-multiply-and-sum image.
 * Replaces DelayAndSumBeamformer._reconstruct_dmas,
 * src/ceep/imaging/beamforming.py:259-313: per pixel the delayed signal of
 * every (tx, rx) pair (k = tx * nant + rx, tx == rx included), then
 * |sum_{k1<k2} s_k1 conj(s_k2)|, normalised like ceep_das.  Same arguments
 * as ceep_das (nant <= 32); work = ceep_dmas_workspace_bytes() bytes.
 * ---------------------------------------------------------------------- */
int64_t ceep_dmas_workspace_bytes(int32_t nx_pix, int32_t ny_pix);
int ceep_dmas(const float* s, const float* kfreq, const float* ant_xy,
              int32_t nfreq, int32_t nant, int32_t nx_pix, int32_t ny_pix,
              float px0, float py0, float pix, int normalize,
              void* work, float* image, void* stream);

/* ------------------------------------------------------------------------
 * Frequency-domain delay-and-sum for callers that cannot allocate device
 * memory.  No counterpart in the reference: it exists for hosts that own all
 * GPU memory through their own pool (for example a scanner pipeline that
 * reserves its memory at start-up and may not allocate mid-scan) and so
 * cannot pass ceep_das a workspace.  Same arguments and result as ceep_das
 * without `work`; the partial sums live in a fixed 2 MiB array inside the
 * library (ceep_das_noalloc_capacity() complex entries) that every GPU which
 * loads the library keeps until exit.  Larger problems are rejected with
 * CEEP_ERR_UNSUPPORTED.  The first call on a device looks up the array's
 * device address (make it before any stream capture).  With lazy module
 * loading (the CUDA 12.2+ default) the array becomes resident only at that
 * first call, so make it before the host reserves its memory pool, or set
 * CUDA_MODULE_LOADING=EAGER.  Calls that overlap on the GPU share the array
 * and race.  The cached address is dropped when a call fails with a CUDA
 * error; no call may follow a device reset without such a failure first.
 * Calls no allocating routine.
 * ---------------------------------------------------------------------- */
int64_t ceep_das_noalloc_capacity(void);
int ceep_das_noalloc(const float* s, const float* kfreq, const float* ant_xy,
                     int32_t nfreq, int32_t nant, int32_t nx_pix, int32_t ny_pix,
                     float px0, float py0, float pix, int normalize,
                     float* image, void* stream);

/* ------------------------------------------------------------------------
 * Time-domain delay-and-sum image.
 * Replaces das_imaging, scripts/verify_dataset_with_das.py:37-103:
 * pixel (i,j) at (i*dx, j*dx); for tx != rx, idx = int((|a_tx-p|+|a_rx-p|)/C/dt)
 * with dt = 1/(4 f) and C = 3e8; image += |s[tx, rx, idx]| when in range.
 * Distances and the index are computed in FP64 with NumPy's rounding sequence
 * (|v| = sqrt(fma(v1, v1, v0*v0))) so the truncation agrees with the
 * reference; |s| is accumulated in FP64.
 *   s      : (nant, nant, ntime) complex64 as float2, s[tx, rx, t]
 *   ant_xy : (nant, 2) double, metres
 *   image  : (grid, grid) float, image[i, j] for pixel (i*dx, j*dx)
 * ---------------------------------------------------------------------- */
int ceep_das_time(const float* s, const double* ant_xy, int32_t nant, int32_t ntime,
                  int32_t grid, double dx, double frequency, float* image, void* stream);

/* ------------------------------------------------------------------------
 * Brain phantom rasteriser for dataset generation.
 * Replaces BrainPhantom2D.get_eps_map with the fixed tissue table
 * (src/ceep/phantoms/head_models.py:519-631, use_gabriel_database=False)
 * and the hemorrhage mask of scripts/generate_corrected_dataset.py:110-118,
 * for `batch` phantoms at once, on the device.
 *   radii   : HOST (5) outer radius in metres of skin, skull, csf, grey, white
 *   tissue  : HOST (6, 2) (eps_r, sigma) of skin, skull, csf, grey, white, blood
 *   hem     : device (batch, 3) hemorrhage centre (metres from the grid centre
 *             cell nx/2, ny/2) and radius; radius < 0 = no hemorrhage
 *   eps_out, sigma_out, mask_out : (batch, nx, ny) FP64 (mask_out may be NULL)
 * Distances are FP64 in the reference's operation order, so every cell lands
 * in the same layer as with NumPy.
 * ---------------------------------------------------------------------- */
int ceep_brain_phantom_2d(int32_t batch, int32_t nx, int32_t ny, double dx, const double* radii,
                          const double* tissue, const double* hem, double* eps_out, double* sigma_out,
                          double* mask_out, void* stream);

/* ------------------------------------------------------------------------
 * 2D update coefficients from the FP64 material maps, on the device.
 * Replaces the host-side coefficient set-up of BatchedFDTD2D
 * (src/ceep/solvers/fdtd_2d_batched.py:151-167, the ADE coefficients of
 * src/ceep/materials/dispersive.py:240-339) with one kernel whose FP64
 * operations follow the host formulas' order with no contraction, so the
 * FP32 results equal the host formulas' bit for bit.
 *   eps_r, sigma : device (nx, ny) FP64 maps (x-major, the reference layout)
 *   poles        : host array of device (nx, ny) FP64 maps, per Debye pole
 *                  (delta_eps, tau), then per Lorentz pole (delta_eps,
 *                  omega_0, delta); n_debye + n_lorentz <= 2
 *   eps0         : the vacuum permittivity the host formulas use
 *   coef         : device (ny, nx, 4) FP32 out: (ca, cb, dt/(eps_r eps0), 0)
 *   ade          : device (poles, ny, nx, 4) FP32 out: Debye (k1, k2,
 *                  (1 + k1)/2, 0), Lorentz (k1, k2, k3, 0); zero where the
 *                  pole's tau / omega_0 is not positive
 * ---------------------------------------------------------------------- */
int ceep2d_material_coefficients(const double* eps_r, const double* sigma, const double* const* poles,
                                 int32_t n_debye, int32_t n_lorentz, int32_t nx, int32_t ny, double dt,
                                 double eps0, float* coef, float* ade, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* CEEP_B200_H */

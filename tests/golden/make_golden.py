"""Generate the golden fixtures in this folder from the reference implementation.

Run in a container that has the reference checkout (path in
CEEP_REFERENCE_ROOT, default /root/reference):

    python tests/golden/make_golden.py            # all fixtures
    python tests/golden/make_golden.py cfg1 ade   # a subset

Every fixture is produced by the reference's own code through ``ref_shim``
(NumPy array module, optional float32 forcing).  Nothing here is used at test
time except the ``.npz`` files it writes.

Fixtures
--------
ceep_results      brain / hemorrhage / empty series from the reference's
                  ceep_results.json (CuPy GPU run, 64x64, 100 steps)
fdtd2d_small_*    BatchedFDTD2D.run(), 48x40, CPML 6, 3 TX, 4 probes, 260 steps,
                  lossy disk; probes + final fields + all eight psi arrays
fdtd2d_cfg1_*     BatchedFDTD2D.run() at 200x200, 8 TX, 400 steps, CPML 15,
                  disk r=40 eps 40 sigma 0.5 (the CPU-runnable headline case)
fdtd2d_runcpu     BatchedFDTD2D.run_cpu() 40x36, 3 TX
fdtd3d_small_*    BatchedFDTD3D.run(), 20^3, CPML 4, 3 TX (two inside the PML
                  shell), region with sigma_m, sphere; probes, fields, psi, energy
dft_cfg1          DFTMonitor over the cfg1 FP64 probe series, 101 frequencies
das_small         DelayAndSumBeamformer DAS and DMAS on a 6-antenna S-matrix
das_time_small    das_imaging (scripts/verify_dataset_with_das.py)
ade2d_small       batched step composed with DispersiveManager (Debye pole 0,
                  Lorentz pole 1), 44x40, CPML 5, 2 TX, 220 steps
single2d          the non-batched FDTD2D (TMz and TEz) with CFS-CPML, PEC and
                  Mur boundaries, Gaussian / modulated / CW sources on every
                  component, circle and region materials (sigma_m too);
                  probes, snapshots, final fields, coefficient maps, waveforms
brain_phantom     BrainPhantom2D.get_eps_map (fixed tissue table) for a
                  head-sized 400x380 grid with and without hemorrhage, and
                  the 64x64 dataset-generator grid; hemorrhage masks as
                  scripts/generate_corrected_dataset.py builds them
head600_ref_*     BatchedFDTD2D.run() at 600x600, 16 TX, 800 steps, CPML 15
                  on the seeded head phantom's non-dispersive maps, FP32
                  and FP64 (about 7 minutes each on one core)
head600_oracle    the oracle (FP64) on the same phantom with its Debye poles:
                  probes, S at 301 frequencies, 64x64 DAS image
head192_oracle    the 3D oracle (FP64) at 192^3, 1000 steps, CPML 10, Debye
                  shells with an inclusion; 4 of the 8 TX (spawn workers)
positions         antenna positions of CircularArray and of the dataset
                  generator's circle
"""
from __future__ import annotations

import contextlib
import io
import json
import os
import sys
import types

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)
from ref_shim import REFERENCE_ROOT, import_reference  # noqa: E402

CFG1 = dict(nx=200, ny=200, dx=0.5e-3, total_steps=400, cpml_thickness=15,
            frequency=2e9)
CFG1_POS = [(int(100 + 70 * np.cos(2 * np.pi * k / 8)), int(100 + 70 * np.sin(2 * np.pi * k / 8)))
            for k in range(8)]
SMALL = dict(nx=48, ny=40, dx=0.5e-3, total_steps=260, cpml_thickness=6, frequency=2e9)
SMALL_SRC = [(20, 18), (8, 30), (40, 6)]
SMALL_PRB = [(20, 18), (7, 7), (41, 33), (24, 2)]


def _probes(out, B, P):
    return np.array([[out[b][p] for p in range(P)] for b in range(B)])


def _save(name, **arrays):
    path = os.path.join(HERE, name + ".npz")
    np.savez_compressed(path, **arrays)
    print("wrote", path, sum(a.nbytes for a in map(np.asarray, arrays.values())), "bytes raw")


def gen_ceep_results():
    with open(os.path.join(REFERENCE_ROOT, "ceep_results.json")) as f:
        d = json.load(f)
    p = d["parameters"]
    sc = d["scenarios"]
    _save("ceep_results",
          empty=np.array(sc["empty"]["signal_real"]),
          brain=np.array(sc["brain"]["signal_real"]),
          hemorrhage=np.array(sc["hemorrhage"]["signal_real"]),
          params=np.array([p["nx"], p["ny"], p["dx"], p["frequency"], p["total_steps"],
                           p["cpml_thickness"], p["antenna_position"][0], p["antenna_position"][1],
                           p["brain_eps_r"], p["brain_sigma"], p["blood_eps_r"], p["blood_sigma"]]))


def gen_small(dtype):
    import_reference(dtype)
    from ceep.solvers.fdtd_2d_batched import BatchedFDTD2D
    s = BatchedFDTD2D(source_positions=SMALL_SRC, probe_positions=SMALL_PRB, **SMALL)
    s.set_material_circle(24, 20, 8, 12.0, 0.3)
    out = s.run()
    names = ["ez", "hx", "hy", "psi_hxy_lo", "psi_hxy_hi", "psi_ezx_lo", "psi_ezx_hi",
             "psi_hyx_lo", "psi_hyx_hi", "psi_ezy_lo", "psi_ezy_hi"]
    _save("fdtd2d_small_" + np.dtype(dtype).name,
          probes=_probes(out, len(SMALL_SRC), len(SMALL_PRB)),
          eps_r=s._eps_r, sigma_e=s._sigma_e, dt=np.float64(s.dt),
          **{k: np.asarray(getattr(s, k)) for k in names})


def gen_cfg1(dtype):
    import_reference(dtype)
    from ceep.solvers.fdtd_2d_batched import BatchedFDTD2D
    s = BatchedFDTD2D(source_positions=CFG1_POS, probe_positions=CFG1_POS, **CFG1)
    s.set_material_circle(100, 100, 40, 40.0, 0.5)
    out = s.run()
    _save("fdtd2d_cfg1_" + np.dtype(dtype).name, probes=_probes(out, 8, 8),
          positions=np.array(CFG1_POS), dt=np.float64(s.dt))


def gen_runcpu():
    import_reference(np.float64)
    from ceep.solvers.fdtd_2d_batched import BatchedFDTD2D
    src = [(10, 12), (30, 20), (19, 30)]
    prb = [(10, 12), (25, 25), (5, 31)]
    s = BatchedFDTD2D(40, 36, 0.5e-3, 150, 5, src, prb, 2e9)
    s.set_material_circle(20, 18, 6, 9.0, 0.2)
    out = s.run_cpu()
    _save("fdtd2d_runcpu", probes=_probes(out, 3, 3), eps_r=s._eps_r, sigma_e=s._sigma_e)


def gen_3d(dtype):
    import_reference(dtype)
    from ceep.solvers.fdtd_3d_batched import BatchedFDTD3D
    src = [(11, 10, 9), (2, 15, 3), (17, 2, 18)]
    prb = [(11, 10, 9), (6, 6, 6), (15, 12, 10), (2, 3, 4)]
    s = BatchedFDTD3D(20, 20, 20, 1e-3, 70, 4, src, prb, 2e9)
    s.set_material_region(8, 14, 7, 13, 6, 12, eps_r=6.0, sigma_e=0.4, mu_r=1.5, sigma_m=200.0)
    s.set_material_sphere(12, 10, 8, 3, eps_r=20.0, sigma_e=1.0)
    out = s.run()
    names = ["ex", "ey", "ez", "hx", "hy", "hz"] + [
        f"psi_{a}_{side}" for a in ("hxy", "hzy", "hyx", "hzx", "hxz", "hyz") for side in ("lo", "hi")]
    _save("fdtd3d_small_" + np.dtype(dtype).name,
          probes=_probes(out, 3, 4), eps_r=s._eps_r, sigma_e=s._sigma_e, mu_r=s._mu_r,
          sigma_m=s._sigma_m, energy=np.float64(s.compute_energy()), dt=np.float64(s.dt),
          src=np.array(src), prb=np.array(prb),
          **{k: np.asarray(getattr(s, k)) for k in names})


def gen_dft():
    import_reference(np.float64)
    from ceep.solvers.dft import DFTMonitor
    d = np.load(os.path.join(HERE, "fdtd2d_cfg1_float64.npz"))
    series, dt = d["probes"], float(d["dt"])
    freqs = np.linspace(0.5e9, 3.5e9, 101)
    mon = DFTMonitor(freqs, (slice(None), slice(None)))
    for step in range(series.shape[2]):
        mon.update(series[:, :, step], step, dt)
    S = mon.get_complex_field().transpose(0, 2, 1)   # (F, rx, tx)
    _save("dft_cfg1", S=S, frequencies=freqs)


def gen_das():
    import_reference(np.float64)
    from ceep.solvers.s_params import MultistaticSParameters
    from ceep.imaging.beamforming import DelayAndSumBeamformer, ImagingRegion
    rng = np.random.default_rng(7)
    N, F = 6, 9
    freqs = np.linspace(1.0e9, 3.0e9, F)
    S = rng.standard_normal((F, N, N)) + 1j * rng.standard_normal((F, N, N))
    ang = 2 * np.pi * np.arange(N) / N
    pos = [(int(40 + 30 * np.cos(a)), int(40 + 30 * np.sin(a))) for a in ang]
    sp = MultistaticSParameters(frequencies=freqs, s_matrix=S, antenna_positions=pos)
    region = ImagingRegion(x_range=(30, 41), y_range=(28, 37), dx=1e-3, background_permittivity=4.0)
    bf = DelayAndSumBeamformer(sp, pos, region, frequency_range=(1.2e9, 2.8e9))
    with contextlib.redirect_stdout(io.StringIO()):
        das = bf.reconstruct("das")
        dmas = DelayAndSumBeamformer(sp, pos, region).reconstruct("dmas")
    _save("das_small", S=S, frequencies=freqs, positions=np.array(pos), das=das, dmas=dmas,
          x_range=np.array(region.x_range), y_range=np.array(region.y_range), dx=np.float64(1e-3),
          eps_bg=np.float64(4.0), frange=np.array([1.2e9, 2.8e9]))


def gen_das_time():
    sys.modules.setdefault("matplotlib", types.ModuleType("matplotlib"))
    sys.modules.setdefault("matplotlib.pyplot", types.ModuleType("matplotlib.pyplot"))
    sys.path.insert(0, os.path.join(REFERENCE_ROOT, "scripts"))
    import verify_dataset_with_das as v
    rng = np.random.default_rng(11)
    N, T, G, dx = 5, 48, 14, 2e-3
    s = rng.standard_normal((N, N, T)) + 1j * rng.standard_normal((N, N, T))
    ang = 2 * np.pi * np.arange(N) / N
    pos = np.stack([0.014 + 0.012 * np.cos(ang), 0.014 + 0.012 * np.sin(ang)], 1)
    img = v.das_imaging(s, pos, 2e9, G, dx)
    _save("das_time_small", s=s, positions=pos, frequency=np.float64(2e9),
          grid_size=np.int64(G), dx=np.float64(dx), image=img)
    # grid-aligned geometry: many delays fall exactly on sample boundaries
    N, T, G, dx = 4, 64, 24, 3.75e-3
    pos = np.array([[0.0, 0.0], [0.0375, 0.0], [0.0, 0.075], [0.0375, 0.0375]])
    s = np.arange(N * N * T, dtype=np.float64).reshape(N, N, T) % 97 + 1.0
    img = v.das_imaging(s.astype(complex), pos, 2e9, G, dx)
    _save("das_time_aligned", s=s, positions=pos, frequency=np.float64(2e9),
          grid_size=np.int64(G), dx=np.float64(dx), image=img)


def gen_ade():
    """Batched step (reference methods) composed with DispersiveManager."""
    import_reference(np.float64)
    from ceep.solvers.fdtd_2d_batched import BatchedFDTD2D
    from ceep.materials.dispersive import DispersiveManager, DebyePole, LorentzPole
    from ceep.core.constants import EPS_0
    nx, ny, n, T = 44, 40, 5, 220
    src = [(14, 20), (30, 12)]
    prb = [(14, 20), (30, 12), (22, 30)]
    s = BatchedFDTD2D(nx, ny, 0.5e-3, T, n, src, prb, 2e9)
    B = len(src)
    x, y = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
    deb_mask = (x - 20) ** 2 + (y - 18) ** 2 <= 7 ** 2
    lor_mask = (x - 27) ** 2 + (y - 24) ** 2 <= 4 ** 2
    s._eps_r[deb_mask] = 8.0
    s._sigma_e[deb_mask] = 0.4
    s._eps_r[lor_mask] = 3.0
    s._sigma_e[lor_mask] = 0.1
    mgrs = []
    for _ in range(B):
        m = DispersiveManager(nx, ny, max_poles=2)
        m.add_poles(deb_mask, [DebyePole(delta_eps=30.0, tau=9e-12)])
        m.add_poles(lor_mask, [DebyePole(delta_eps=0.0, tau=0.0),
                               LorentzPole(delta_eps=5.0, omega_0=2 * np.pi * 6e9, delta=2 * np.pi * 0.5e9)])
        mgrs.append(m)
    s._build()
    dt = s.dt
    eps_add = np.asarray(mgrs[0].compute_coefficients(dt))
    for m in mgrs[1:]:
        m.compute_coefficients(dt)
    # Grid2D._precompute_coefficients (src/ceep/core/grid.py:174-189) with eps_inf = _eps_r
    eps = s._eps_r * EPS_0 + eps_add
    sd = s._sigma_e * dt / (2.0 * eps)
    s.ca = ((1.0 - sd) / (1.0 + sd))[None]
    s.cb = ((dt / eps) / (1.0 + sd))[None]
    P = len(prb)
    probes = np.zeros((B, P, T))
    inv = s.inv_dx
    for step in range(T):
        # interior H and H-CPML: fdtd_2d_batched.py:471-486
        s.hx[:, n:nx - n, n:ny - 1] = (s.da[:, n:nx - n, n:ny - 1] * s.hx[:, n:nx - n, n:ny - 1]
                                       - s.db[:, n:nx - n, n:ny - 1] * inv * (s.ez[:, n:nx - n, n + 1:ny] - s.ez[:, n:nx - n, n:ny - 1]))
        s.hy[:, n:nx - 1, n:ny - n] = (s.da[:, n:nx - 1, n:ny - n] * s.hy[:, n:nx - 1, n:ny - n]
                                       + s.db[:, n:nx - 1, n:ny - n] * inv * (s.ez[:, n + 1:nx, n:ny - n] - s.ez[:, n:nx - 1, n:ny - n]))
        s._apply_h_cpml()
        I = (slice(None), slice(n + 1, nx - n), slice(n + 1, ny - n))
        ez_old = s.ez.copy()
        sum_gj = np.stack([np.asarray(m.get_sum_gamma_j("Ez")) for m in mgrs])
        s.ez[I] = (s.ca[I[0:1] + I[1:]] * s.ez[I] + s.cb[(slice(None),) + I[1:]] * (
            (s.hy[I] - s.hy[:, n:nx - n - 1, n + 1:ny - n]) * inv
            - (s.hx[I] - s.hx[:, n + 1:nx - n, n:ny - n - 1]) * inv))
        s.ez[I] -= s.cb[(slice(None),) + I[1:]] * sum_gj[I]
        for b, m in enumerate(mgrs):
            m.update_j_fields("Ez", s.ez[b], ez_old[b], dt)
        s._apply_e_cpml()
        s.ez[:, 0, :] = 0
        s.ez[:, -1, :] = 0
        s.ez[:, :, 0] = 0
        s.ez[:, :, -1] = 0
        w = float(s.waveform[step])
        for b in range(B):
            s.ez[b, src[b][0], src[b][1]] += w
        for p, (px, py) in enumerate(prb):
            probes[:, p, step] = s.ez[:, px, py]
    _save("ade2d_small", probes=probes, eps_r=s._eps_r, sigma_e=s._sigma_e,
          deb_mask=deb_mask, lor_mask=lor_mask, ez=s.ez,
          j0=np.stack([np.asarray(m.j_ez[0]) for m in mgrs]),
          j1=np.stack([np.asarray(m.j_ez[1]) for m in mgrs]))


def gen_brain_phantom():
    """BrainPhantom2D maps and the dataset generator's hemorrhage mask."""
    import_reference(np.float64)
    from ceep.phantoms import BrainPhantom2D
    cases = [  # nx, ny, dx, hemorrhage (cm) or None, radius (cm), head radius (cm)
        (400, 380, 0.5e-3, (2.1, -1.3), 1.2, 9.0),
        (400, 380, 0.5e-3, None, 1.0, 9.0),
        (64, 64, 0.5e-3, (0.4, -0.25), 0.6, 9.0),
        (90, 70, 1e-3, (-0.9, 0.7), 0.45, 4.0),
    ]
    out = {}
    for k, (nx, ny, dx, loc, rad, head) in enumerate(cases):
        ph = BrainPhantom2D(nx=nx, ny=ny, dx=dx, hemorrhage_location=loc, hemorrhage_radius=rad,
                            head_radius_cm=head, use_gabriel_database=False)
        eps, sig = ph.get_eps_map(2e9)
        mask = np.zeros((nx, ny))
        if loc is not None:  # generate_corrected_dataset.py:110-118
            cx, cy = nx // 2, ny // 2
            xg, yg = np.meshgrid(np.arange(nx), np.arange(ny), indexing="ij")
            r = np.sqrt(((xg - cx) * dx - loc[0] * 1e-2) ** 2 + ((yg - cy) * dx - loc[1] * 1e-2) ** 2)
            mask[r <= rad * 1e-2] = 1.0
        out[f"eps_{k}"], out[f"sigma_{k}"], out[f"mask_{k}"] = eps, sig, mask
        out[f"case_{k}"] = np.array([nx, ny, dx, np.nan if loc is None else loc[0],
                                     np.nan if loc is None else loc[1], rad, head])
    _save("brain_phantom", **out)


# non-batched FDTD2D cases: (name, mode, nx, ny, steps, boundaries, sources, probes,
# record_field, record_interval, materials)
SINGLE2D = [
    ("tmz_cpml", "TMZ", 64, 56, 320,
     [("cpml", 8, 4, 2.0, 0.05, 1.0)],
     [("gauss", 30, 24, 20e9, 1.0, 6.0, "Ez"), ("modgauss", 4, 30, 8e9, 20e9, 0.5, 5.0, "Ez"),
      ("gauss", 40, 40, 20e9, 1.0, 6.0, "Hz")],
     [(30, 24), (50, 44), (3, 10), (62, 54)], "Ez", 40,
     [("circle", 34, 28, 7, 4.0, 1.0, 0.2, 0.0), ("region", 10, 20, 36, 48, 2.5, 1.0, 0.05, 0.0)]),
    ("tez_cpml", "TEZ", 60, 52, 300,
     [("cpml", 6, 3, 1.5, 0.1, 2.0)],
     [("gauss", 28, 26, 20e9, 1.0, 6.0, "Hz"), ("gauss", 20, 30, 15e9, 0.7, 5.0, "Ex"),
      ("sin", 36, 18, 12e9, 0.3, "Ey"), ("gauss", 33, 33, 20e9, 1.0, 6.0, "Ez")],
     [(28, 26), (45, 40), (2, 2), (58, 25)], "Hz", 50,
     [("circle", 30, 26, 6, 5.0, 1.0, 0.3, 0.0), ("region", 40, 50, 10, 20, 1.0, 2.0, 0.0, 300.0)]),
    ("tmz_pec", "TMZ", 40, 36, 220, [("pec",)],
     [("gauss", 12, 20, 20e9, 1.0, 6.0, "Ez")], [(12, 20), (30, 10), (0, 5)], "Ez", 55,
     [("circle", 22, 18, 5, 6.0, 1.0, 0.1, 0.0)]),
    ("tmz_mur", "TMZ", 42, 38, 240, [("mur",)],
     [("gauss", 20, 19, 20e9, 1.0, 6.0, "Ez")], [(20, 19), (35, 30), (0, 0), (41, 10)], None, 1,
     [("region", 5, 15, 5, 15, 3.0, 1.0, 0.0, 0.0)]),
    ("tez_pec_cpml", "TEZ", 48, 44, 260, [("pec",), ("cpml", 7, 4, 2.0, 0.05, 1.0)],
     [("gauss", 24, 22, 20e9, 1.0, 6.0, "Hz")], [(24, 22), (10, 35), (47, 43)], "Ey", 65,
     [("circle", 24, 22, 5, 3.0, 1.0, 0.0, 0.0)]),
    ("tez_mur", "TEZ", 40, 40, 200, [("mur",)],
     [("gauss", 18, 21, 20e9, 1.0, 6.0, "Hz")], [(18, 21), (39, 39), (1, 20)], "Hz", 40, []),
]


def gen_single2d():
    """The reference's own non-batched FDTD2D (TMz/TEz) with CPML, PEC and Mur
    boundaries, mixed sources and materials; probes, snapshots, final fields."""
    import_reference(np.float64)
    from ceep.boundaries.absorbing import CPML, PEC, MurABC
    from ceep.core.config import GridConfig, SimulationConfig, SimulationMode
    from ceep.solvers.fdtd_2d import FDTD2D
    from ceep.sources.waveforms import GaussianSource, ModulatedGaussianSource, SinusoidalSource
    out = {}
    for name, mode, nx, ny, steps, bcs, srcs, prbs, rec, interval, mats in SINGLE2D:
        cfg = SimulationConfig(grid=GridConfig(nx=nx, ny=ny, dx=1e-3, dy=0.8e-3),
                               mode=getattr(SimulationMode, mode), total_steps=steps)
        boundaries = []
        for b in bcs:
            if b[0] == "cpml":
                boundaries.append(CPML(thickness=b[1], order=b[2], sigma_factor=b[3], alpha_max=b[4],
                                       kappa_max=b[5]))
            elif b[0] == "mur":
                boundaries.append(MurABC())
            else:
                boundaries.append(PEC())
        sources = []
        for sp in srcs:
            if sp[0] == "gauss":
                sources.append(GaussianSource(x=sp[1], y=sp[2], frequency_max=sp[3], amplitude=sp[4],
                                              delay_factor=sp[5], field_component=sp[6]))
            elif sp[0] == "modgauss":
                sources.append(ModulatedGaussianSource(x=sp[1], y=sp[2], frequency=sp[3], bandwidth=sp[4],
                                                       amplitude=sp[5], delay_factor=sp[6],
                                                       field_component=sp[7]))
            else:
                sources.append(SinusoidalSource(x=sp[1], y=sp[2], frequency=sp[3], amplitude=sp[4],
                                                field_component=sp[5]))
        s = FDTD2D(cfg, sources=sources, boundaries=boundaries, record_field=rec, record_interval=interval,
                   probe_points=[tuple(p) for p in prbs])
        for m in mats:
            if m[0] == "circle":
                s.grid.set_material_circle(m[1], m[2], m[3], eps_r=m[4], mu_r=m[5], sigma_e=m[6], sigma_m=m[7])
            else:
                s.grid.set_material_region(m[1], m[2], m[3], m[4], eps_r=m[5], mu_r=m[6], sigma_e=m[7],
                                           sigma_m=m[8])
        s.grid._precompute_coefficients()
        # on the NumPy array module the reference's snapshots alias the live
        # field (to_numpy returns the array itself), so every entry ends up as
        # the final state; the snapshots kept here are copies taken after the
        # reference's own step() at the steps its _record() would use
        snaps = []
        for n in range(steps):
            s.step()
            if rec and n % interval == 0:
                snaps.append(np.array(s.get_field(rec)))
        g = s.grid
        fields = ("ez", "hx", "hy") if mode == "TMZ" else ("hz", "ex", "ey")
        out[name + "_probes"] = np.array([s.probe_data[tuple(p)] for p in prbs])
        out[name + "_snapshots"] = np.array(snaps) if snaps else np.zeros((0, nx, ny))
        for f in fields:
            out[f"{name}_{f}"] = np.asarray(getattr(g, f))
        for k in ("_ca", "_cb", "_da", "_db"):
            out[name + k] = np.asarray(getattr(g, k))
        out[name + "_dt"] = np.float64(cfg.dt)
        out[name + "_waveforms"] = np.array([[src.value_at(n, cfg.dt) for n in range(steps)] for src in sources])
    _save("single2d", **out)


# Full-size cases at the benchmarked configurations.  Their inputs are the
# seeded synthetic phantoms of ceep_b200.phantoms (pure NumPy); the SHA-256 of
# every input map is stored with the outputs, so a test can tell a changed
# phantom generator from a changed solver.
HEAD600 = dict(nx=600, ny=600, dx=0.5e-3, total_steps=800, cpml_thickness=15, frequency=2e9)
HEAD600_SEED = 1000
HEAD600_FREQS = (0.5e9, 3.5e9, 301)
HEAD600_DAS = dict(npix=64, half=0.09)        # 64x64 pixels over +/-9 cm around the centre
HEAD192 = dict(nx=192, ny=192, nz=192, dx=1e-3, total_steps=1000, cpml_thickness=10, frequency=2e9)
HEAD192_SEED = 1000
HEAD192_TX = (0, 3, 5, 6)                     # both float4 lanes of the 8-TX layout


def _sha(*arrays):
    import hashlib
    h = hashlib.sha256()
    for a in arrays:
        h.update(np.ascontiguousarray(np.asarray(a, np.float64)).tobytes())
    return h.hexdigest()


def _head600_inputs():
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from ceep_b200.phantoms import HeadPhantom2D, ring_positions
    c = HEAD600["nx"] // 2
    pos = ring_positions(16, (c, c), 200)
    ph = HeadPhantom2D(HEAD600["nx"], HEAD600["ny"], HEAD600["dx"], seed=HEAD600_SEED)
    eps, sig = ph.get_eps_map()
    (de, tau), = ph.get_dispersion()["debye"]
    return pos, eps, sig, de, tau


def gen_head600_ref(dtype):
    """The reference's own BatchedFDTD2D.run() at the head-imaging size (600^2,
    16 TX on a ring of radius 200 cells, 800 steps, CPML 15) on the seeded head
    phantom's non-dispersive maps (eps_inf, sigma written to _eps_r/_sigma_e,
    as the reference's callers do): the batched reference has no ADE."""
    pos, eps, sig, _, _ = _head600_inputs()
    import_reference(dtype)
    from ceep.solvers.fdtd_2d_batched import BatchedFDTD2D
    s = BatchedFDTD2D(source_positions=pos, probe_positions=pos, **HEAD600)
    s._eps_r[:] = eps
    s._sigma_e[:] = sig
    out = s.run()
    _save("head600_ref_" + np.dtype(dtype).name, probes=_probes(out, 16, 16).astype(dtype),
          positions=np.array(pos), dt=np.float64(s.dt), inputs_sha=np.array(_sha(eps, sig)))


def gen_head600_oracle():
    """Config 2 proper from the oracle (FP64): the same phantom with its Debye
    pole per layer; probe series, S at 301 frequencies and the 64x64 DAS image."""
    pos, eps, sig, de, tau = _head600_inputs()
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from oracle.fdtd2d import Fdtd2DOracle
    from oracle.spectral import das_frequency, running_dft
    o = Fdtd2DOracle(HEAD600["nx"], HEAD600["ny"], HEAD600["dx"], HEAD600["total_steps"],
                     HEAD600["cpml_thickness"], pos, pos, HEAD600["frequency"], eps_r=eps, sigma_e=sig,
                     dispersion={"debye": [(de, tau)]})
    probes = o.run()
    freqs = np.linspace(*HEAD600_FREQS)
    S = running_dft(probes, o.dt, freqs)
    npix, half, dx = HEAD600_DAS["npix"], HEAD600_DAS["half"], HEAD600["dx"]
    pitch = 2 * half / npix
    x0 = ((HEAD600["nx"] // 2) * dx - half) / pitch
    y0 = ((HEAD600["ny"] // 2) * dx - half) / pitch
    ant = np.asarray(pos, np.float64) * dx / pitch   # grid index -> pitch units
    img = das_frequency(S, freqs, ant, (x0, x0 + npix), (y0, y0 + npix), pitch)
    _save("head600_oracle", probes=probes, S=S, das=img, positions=np.array(pos), dt=np.float64(o.dt),
          inputs_sha=np.array(_sha(eps, sig, de, tau)))


def _head192_inputs():
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))
    from ceep_b200.phantoms import HeadPhantom3D, ring_positions
    c = HEAD192["nx"] // 2
    pos = [(x, y, HEAD192["nz"] // 2) for x, y in ring_positions(8, (c, c), 75)]
    ph = HeadPhantom3D(HEAD192["nx"], HEAD192["ny"], HEAD192["nz"], HEAD192["dx"], seed=HEAD192_SEED)
    eps, sig = ph.get_eps_map_3d()
    (de, tau), = ph.get_dispersion()["debye"]
    return pos, eps, sig, de, tau


def _head192_one_tx(tx):
    pos, eps, sig, de, tau = _head192_inputs()
    from oracle.fdtd3d import Fdtd3DOracle
    o = Fdtd3DOracle(HEAD192["nx"], HEAD192["ny"], HEAD192["nz"], HEAD192["dx"], HEAD192["total_steps"],
                     HEAD192["cpml_thickness"], [pos[tx]], pos, HEAD192["frequency"], eps_r=eps, sigma_e=sig,
                     dispersion={"debye": [(de, tau)]})
    return o.run()[0]


def gen_head192_oracle():
    """Config 5's forward from the 3D oracle (FP64): 192^3, 1 mm, 1000 steps,
    CPML 10, 8 Ez dipoles on a mid-plane ring, seeded Debye ellipsoid shells
    with an inclusion.  The transmit events are independent, so four of the
    eight (both float4 lanes) run in parallel worker processes."""
    import multiprocessing as mp
    pos, eps, sig, de, tau = _head192_inputs()
    with mp.get_context("spawn").Pool(len(HEAD192_TX)) as pool:
        rows = pool.map(_head192_one_tx, HEAD192_TX)
    from oracle.fdtd3d import reference_dt_3d
    _save("head192_oracle", probes=np.stack(rows), tx=np.array(HEAD192_TX), positions=np.array(pos),
          dt=np.float64(reference_dt_3d(HEAD192["dx"])), inputs_sha=np.array(_sha(eps, sig, de, tau)))


# CircularArray cases: (num_antennas, radius_mm, center, dx)
CIRCULAR = [(8, 35.0, (100, 100), 0.5e-3), (16, 100.0, (300, 300), 0.5e-3), (12, 70.0, (100, 100), 1e-3),
            (24, 120.0, (200, 200), 1e-3), (16, 75.0, (96, 96, 96), 1e-3), (8, 75.0, (96, 96, 96), 1e-3)]
DATASET_GRIDS = [(64, 8), (64, 16), (128, 16), (256, 12), (600, 16)]   # (nx = ny, n_ant)


def gen_positions():
    """Antenna grid positions from the reference's CircularArray
    (src/ceep/antennas/arrays.py:110-143) and from its dataset generator's
    circle (scripts/generate_corrected_dataset.py:121-129), the latter read off
    the source positions generate_sample() hands the solver (a stand-in
    solver class records them and stops the sample)."""
    import_reference(np.float64)
    from ceep.antennas.arrays import CircularArray
    out = {}
    for k, (n, rmm, c, dx) in enumerate(CIRCULAR):
        out[f"circular_{k}"] = np.array([e.position for e in CircularArray(n, rmm, c, dx).elements])
        out[f"circular_case_{k}"] = np.array([n, rmm, dx] + list(c) + ([0] if len(c) == 2 else []), np.float64)
    sys.path.insert(0, os.path.join(REFERENCE_ROOT, "scripts"))
    import generate_corrected_dataset as gcd

    class _Stop(Exception):
        pass

    class _Recorder:
        def __init__(self, **kw):
            raise _Stop(kw["source_positions"])

    gcd.BatchedFDTD2D = _Recorder
    for k, (nx, n_ant) in enumerate(DATASET_GRIDS):
        try:
            with contextlib.redirect_stdout(io.StringIO()):
                gcd.generate_sample(0, include_hemorrhage=False, nx=nx, ny=nx, n_ant=n_ant)
        except _Stop as e:
            out[f"dataset_{k}"] = np.array(e.args[0])
        out[f"dataset_case_{k}"] = np.array([nx, n_ant])
    _save("positions", **out)


JOBS = {
    "positions": gen_positions,
    "head600_ref32": lambda: gen_head600_ref(np.float32),
    "head600_ref64": lambda: gen_head600_ref(np.float64),
    "head600_oracle": gen_head600_oracle,
    "head192_oracle": gen_head192_oracle,
    "single2d": gen_single2d,
    "ceep_results": gen_ceep_results,
    "brain_phantom": gen_brain_phantom,
    "small": lambda: (gen_small(np.float64), gen_small(np.float32)),
    "cfg1": lambda: (gen_cfg1(np.float64), gen_cfg1(np.float32)),
    "runcpu": gen_runcpu,
    "3d": lambda: (gen_3d(np.float64), gen_3d(np.float32)),
    "dft": gen_dft,
    "das": gen_das,
    "das_time": gen_das_time,
    "ade": gen_ade,
}

if __name__ == "__main__":
    sys.path.insert(0, os.path.dirname(os.path.dirname(HERE)))  # oracle/ for the spawn workers
    for job in (sys.argv[1:] or list(JOBS)):
        JOBS[job]()

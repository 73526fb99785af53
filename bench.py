#!/usr/bin/env python3
"""Throughput of the batched multistatic FDTD path on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--workload head600|disk200|head192|pack256|adjoint400|adjoint192|single4096]

A bench "step" is one complete head-imaging sample: the 800-step fused FDTD
time loop for 16 transmit events with a one-pole Debye phantom, the DFT of
all 16x16 probe series into S (301 frequencies) and a 64x64 DAS image.
Metric: GCell-steps/s = nx * ny * time steps * TX / time.

Multi-GPU: phantoms are independent, so each rank runs its own samples
(weak scaling, no data-path collective); time is the max over ranks.

The reference arm (--impl reference) times the CPU restatement of the
reference algorithm (the oracle, NumPy FP64) on the host cores, spreading the
transmit events over worker processes, on a bounded number of time steps.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOADS = {
    # config 2 of the headline metric: 600x600, 0.5 mm, 800 steps, CPML 15, 16 TX/RX
    # on r = 200 cells, Debye head phantom, 301 frequencies, 64x64 DAS
    "head600": dict(nx=600, ny=600, dx=0.5e-3, steps=800, cpml=15, ntx=16, ring=200, nfreq=301, das=64,
                    debye=True),
    # config 1 (the reference's CPU-runnable case): 200x200, 400 steps, 8 TX, disk
    "disk200": dict(nx=200, ny=200, dx=0.5e-3, steps=400, cpml=15, ntx=8, ring=70, nfreq=101, das=64,
                    debye=False),
    # config 5: 192^3, 1 mm, 1000 steps, CPML 10, 8 z-directed TX/RX on a mid-plane
    # ring, Debye ellipsoid shells with an inclusion, 101 frequencies
    "head192": dict(dim=3, nx=192, ny=192, nz=192, dx=1e-3, steps=1000, cpml=10, ntx=8, ring=75, nfreq=101,
                    das=64, debye=True),
}
PUBLISHED_GCELLS = 1.40  # README.md:60 of the reference: 600x600x16 TX x 800 steps in 3.3 s (T4)


def algorithmic_bytes_per_step(w, n_debye):
    if w.get("dim", 2) == 3:
        return algorithmic_bytes_per_step_3d(w, n_debye)
    return algorithmic_bytes_per_step_2d(w, n_debye)


def algorithmic_bytes_per_step_3d(w, n_debye):
    """Compulsory FP32 DRAM bytes of one 3D step: 48 B per cell-TX (six field
    components read and written once), 16 B per cell for (da, db, ca, cb),
    16 B per face cell-TX for its two psi, and per Debye pole 24 B per
    interior cell-TX (three currents) plus 12 B per interior cell."""
    nx, ny, nz, n, T = w["nx"], w["ny"], w["nz"], w["cpml"], w["ntx"]
    cells = nx * ny * nz
    faces = 2 * n * (ny * nz + nx * nz + nx * ny)
    interior = (nx - 2 * n - 1) * (ny - 2 * n - 1) * (nz - 2 * n - 1)
    return cells * (48 * T + 16) + faces * 16 * T + n_debye * interior * (24 * T + 12)


def algorithmic_bytes_per_step_2d(w, n_debye, n_lorentz=0):
    """Compulsory FP32 DRAM bytes of one fused step (read+write each state word
    once, coefficients once per cell): 24 B per cell-TX for Ez/Hx/Hy, 8 B per
    cell for (ca, cb), 16 B per strip cell-TX for the H and E psi of that
    strip plus 4 B per strip cell for dt/eps, and per Debye pole 8 B per
    interior cell-TX for J plus 12 B per interior cell for (k1, k2, gamma)."""
    nx, ny, n, T = w["nx"], w["ny"], w["cpml"], w["ntx"]
    cells = nx * ny
    xstrip = 2 * n * ny
    ystrip = 2 * n * nx
    interior = (nx - 2 * n - 1) * (ny - 2 * n - 1)
    b = cells * (24 * T + 8)
    b += (xstrip + ystrip) * (16 * T + 4)
    b += n_debye * interior * (8 * T + 12)
    b += n_lorentz * interior * (16 * T + 12)   # J and J_prev read+write, (k1, k2, k3)
    return b


# CUDA sources a kernel's DRAM traffic depends on (their hash is recorded in
# the profile summary the traffic figure comes from)
KERNEL_SOURCES = {2: ("fdtd2d.cu", "fdtd2d.cuh", "fdtd2d_kernels.cuh", "common.cuh", "tma.cuh"),
                  3: ("fdtd3d.cu", "fdtd3d.cuh", "common.cuh")}


def kernel_source_sha(dim):
    import hashlib
    h = hashlib.sha256()
    for f in KERNEL_SOURCES[dim]:
        with open(os.path.join(ROOT, "ceep_b200", "csrc", f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def profile_traffic(name, dim):
    """(DRAM bytes per launch, provenance) from the committed ncu summary
    profiles/<name>: the `dram_bytes_per_launch = N` line, and whether its
    `source_sha256 = ...` line matches the kernel sources built now."""
    path = os.path.join(ROOT, "profiles", name)
    if not os.path.exists(path):
        return None, None
    traffic, sha, rows = None, None, None
    for line in open(path):
        if line.startswith("dram_bytes_per_launch"):
            traffic = int(line.split("=")[1])
        elif line.startswith("source_sha256"):
            sha = line.split("=")[1].strip()
        elif line.startswith("tile_rows"):
            rows = int(line.split("=")[1])
    return traffic, {"file": "profiles/" + name, "source_sha256": sha, "tile_rows": rows,
                     "matches_current_source": sha == kernel_source_sha(dim) if sha else None}


def hbm_peak():
    """(GB/s, source): the measured copy bandwidth of MEASURED_PEAKS.json, else
    the pool's earlier measurement (6650 GB/s)."""
    peaks_path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(peaks_path):
        return json.load(open(peaks_path))["hbm_gbs"], "measured"
    return 6650.0, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = []
        for line in (self.out or "").strip().splitlines():
            f = [v.strip() for v in line.split(",")]
            if len(f) >= 9:
                rows.append(f)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i, v in enumerate(r[5:9]) if v.strip().lower() == "active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def build_inputs_3d(w, nsamples, device, seed0=1000):
    from ceep_b200 import BatchedFDTD3D
    from ceep_b200.phantoms import HeadPhantom3D, ring_positions
    c = w["nx"] // 2
    pos = [(x, y, w["nz"] // 2) for x, y in ring_positions(w["ntx"], (c, w["ny"] // 2), w["ring"])]
    freqs = np.linspace(0.5e9, 3.5e9, w["nfreq"])
    solver = BatchedFDTD3D(w["nx"], w["ny"], w["nz"], w["dx"], w["steps"], w["cpml"], pos, pos, 2e9,
                           frequencies=freqs, device=str(device))
    phantoms, mats = [], []
    for k in range(nsamples):
        sc = min(w["nx"], w["ny"], w["nz"]) / 192.0           # shells scaled to the grid
        ph = HeadPhantom3D(w["nx"], w["ny"], w["nz"], w["dx"], seed=seed0 + k,
                           semi_axes=(0.070 * sc, 0.056 * sc, 0.060 * sc))
        eps, sig = ph.get_eps_map_3d()
        d = ph.get_dispersion()
        mats.append(solver.material_tensors(eps, sig, d["debye"], d["lorentz"]))
        phantoms.append(ph)
    solver.set_phantom(phantoms[0])
    return solver, pos, freqs, phantoms, mats


def build_inputs(w, nsamples, device, seed0=1000):
    if w.get("dim", 2) == 3:
        return build_inputs_3d(w, nsamples, device, seed0)
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.phantoms import HeadPhantom2D, ring_positions
    pos = ring_positions(w["ntx"], (w["nx"] // 2, w["ny"] // 2), w["ring"])
    freqs = np.linspace(0.5e9, 3.5e9, w["nfreq"])
    solver = BatchedFDTD2D(w["nx"], w["ny"], w["dx"], w["steps"], w["cpml"], pos, pos, 2e9,
                           frequencies=freqs, device=str(device))
    phantoms, mats = [], []
    for k in range(nsamples):
        if w["debye"]:
            ph = HeadPhantom2D(w["nx"], w["ny"], w["dx"], seed=seed0 + k)
            eps, sig = ph.get_eps_map()
            d = ph.get_dispersion()
            mats.append(solver.material_tensors(eps, sig, d["debye"], d["lorentz"]))
        else:
            x, y = np.meshgrid(np.arange(w["nx"]), np.arange(w["ny"]), indexing="ij")
            m = (x - w["nx"] // 2) ** 2 + (y - w["ny"] // 2) ** 2 <= 40 ** 2
            ph = None
            mats.append(solver.material_tensors(np.where(m, 40.0, 1.0), np.where(m, 0.5, 0.0)))
        phantoms.append(ph)
    if w["debye"]:
        solver.set_phantom(phantoms[0])
    else:
        solver.set_material_circle(w["nx"] // 2, w["ny"] // 2, 40, 40.0, 0.5)
    return solver, pos, freqs, phantoms, mats


def one_sample(solver, w, freqs, pos, das_ws, stream):
    """Device-only sample: fresh state, the time loop, S, DAS image."""
    import torch
    from ceep_b200.spectral import das_image, dft
    solver.reset()
    solver.advance(0, w["steps"], stream=stream)
    S = dft(solver.probe_data, freqs, solver.dt)
    half = 0.09 if w.get("dim", 2) == 2 else 0.07
    img = das_image(S, freqs, np.asarray([p[:2] for p in pos], float) * w["dx"], w["das"], w["das"],
                    (w["nx"] // 2) * w["dx"] - half, (w["ny"] // 2) * w["dx"] - half, 2 * half / w["das"],
                    299_792_458.0, True, workspace=das_ws)
    return S, img


def run_ours(args, w):
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=120), device_id=torch.device("cuda", local))
    device = torch.device("cuda", local)
    torch.cuda.set_device(device)
    K, W = args.steps, args.warmup
    solver, pos, freqs, phantoms, mats = build_inputs(w, K + W, device, seed0=1000 + 97 * rank)
    tblock = apply_temporal_block(solver, w, args.temporal_block)
    solver._build()
    tile_rows = None
    if w.get("dim", 2) == 2 and not args.no_autotune:
        solver.load_material_tensors(mats[0])
        solver.autotune()                  # tile height for this grid (results do not depend on it)
        tile_rows = solver.rows_per_block
    stream = torch.cuda.current_stream(device)
    das_ws = torch.empty(1 << 20, dtype=torch.uint8, device=device)
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=device)  # > 126 MB L2
    n_debye = 1 if w["debye"] else 0

    for k in range(W):
        solver.load_material_tensors(mats[K + k])
        one_sample(solver, w, freqs, pos, das_ws, stream)
    torch.cuda.synchronize()

    # -- timed region: K samples, inputs resident in HBM, L2 flushed between samples
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(K)]
    if world > 1:
        dist.barrier()
    torch.cuda.synchronize()
    with ClockSampler(local) as clk:
        for k in range(K):
            flush.zero_()
            solver.load_material_tensors(mats[k])
            ev[k][0].record(stream)
            one_sample(solver, w, freqs, pos, das_ws, stream)
            ev[k][1].record(stream)
        torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    ms = [a.elapsed_time(b) for a, b in ev]
    total_ms = float(np.sum(ms))
    if world > 1:
        from ceep_b200.distributed import max_time_ms
        total_ms = max_time_ms(total_ms, device)
    cell_steps = w["nx"] * w["ny"] * w.get("nz", 1) * w["steps"] * w["ntx"]
    value = world * K * cell_steps / (total_ms * 1e-3) / 1e9

    # -- dominant kernel alone: the fused step kernel (one or two steps per
    # launch), per-launch time over full loops.  Algorithmic bytes per launch
    # = the unblocked per-cell-step formula x the cell-steps one launch
    # advances (two steps for the temporally blocked kernel, which reads and
    # writes the state once for both: its DRAM traffic is below that figure,
    # reported separately as dram_gbs)
    launches = solver.launches(w["steps"]) if w.get("dim", 2) == 2 else w["steps"]   # kernels
    blocks = (w["steps"] + tblock - 1) // tblock if w.get("dim", 2) == 2 else w["steps"]  # time-step blocks
    per_launch = []
    for k in range(3):
        flush.zero_()
        solver.reset()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        solver.advance(0, w["steps"], stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        per_launch.append(a.elapsed_time(b) / blocks)
    launch_ms = float(np.median(per_launch))
    bytes_step = algorithmic_bytes_per_step(w, n_debye)
    peak, peak_src = hbm_peak()
    steps_per_launch = tblock if w.get("dim", 2) == 2 else 1
    bytes_launch = bytes_step * steps_per_launch
    achieved = bytes_launch / (launch_ms * 1e-3) / 1e9
    kname = "fdtd3d_kernels" if w.get("dim", 2) == 3 else ("fdtd2d_step2" if tblock == 2 else "fdtd2d_step")
    traffic, traffic_src = profile_traffic(f"{kname}_{args.workload}.md", w.get("dim", 2))

    # -- end to end through the public API with host buffers
    e2e = None
    if not args.no_e2e:
        e2e = run_e2e(w, phantoms[:min(K, 5)], pos, freqs, device, tblock, rows=tile_rows or 0)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_baseline(w, sample_steps=args.cpu_steps if w.get("dim", 2) == 2 else 2)

    # config 4's gradient cost (outside the timed region, one GPU only): the
    # checkpointed adjoint at K = 50 and every step kept, against one forward
    grad4 = pack3 = fwd5 = None
    if rank == 0 and world == 1 and args.workload == "head600" and not args.no_secondary:
        t_fwd, ratios, _, _, _ = adjoint400_ratios(Ks=(1, 50), keep_budget=0, reps=2, split=False)
        grad4 = {"workload": "adjoint400 (400^2, 1000 steps, 16 TX, Debye, S misfit)",
                 "forward_ms": round(t_fwd, 3),
                 "gradient_x_forward": {f"K={k}": round(v, 3) for k, v in ratios.items()}}
        # config 3's packed uneven batch (256 seeded phantoms, one timed run)
        del solver
        torch.cuda.empty_cache()
        m = pack_measure(256, 32, 1)
        pack3 = {"workload": "pack256 (256 phantoms 256..768^2, 600..1200 steps, 8..16 TX, 1/3 Lorentz)",
                 "value": round(m["value"], 3), "unit": "GCell-steps/s",
                 "roofline_frac": round(m["achieved"] / m["peak"], 3),
                 "speedup_vs_run": round(m["value"] / m["base_fresh"], 2),
                 "speedup_vs_replay": round(m["value"] / m["base_replay"], 2),
                 "tile_rows": m["pk"].rows, "temporal_block": m["pk"].temporal_block}
        del m
        torch.cuda.empty_cache()
        fwd5 = head192_forward_figure()

    if world > 1:
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": "batched FDTD GCell-steps/s", "value": round(value, 3), "unit": "GCell-steps/s",
        "n_gpus": world, "steps": K, "warmup": W, "ms_per_step": round(total_ms / K, 3),
        "higher_is_better": True, "scaling": "weak",
        "vs_baseline": round(value / PUBLISHED_GCELLS, 2) if args.workload == "head600" else None,
        "dtype": "f32", "data": "synthetic (seeded phantoms)",
        "config": {"workload": args.workload, "nx": w["nx"], "ny": w["ny"], "nz": w.get("nz", 1),
                   "time_steps": w["steps"],
                   "tx": w["ntx"], "cpml": w["cpml"], "debye_poles": n_debye, "dft_freqs": w["nfreq"],
                   "das": f"{w['das']}x{w['das']}", "parallelism": f"replicas{world}",
                   "tile_rows": tile_rows if tile_rows else "automatic",
                   "l2": "flushed (256 MB write) before every sample; per-step working set > L2",
                   "sample": "fused time loop + DFT->S + DAS image"},
        "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                     "frac": round(achieved / peak, 3), "traffic": traffic, "traffic_source": traffic_src,
                     "peak_source": peak_src,
                     "kernel": (("fdtd2d_step2_kernel (two steps per launch)" if tblock == 2 else
                                 "fdtd2d_step_kernel") if w.get("dim", 2) == 2 else
                                "fdtd3d step: h box + h shell (side stream) + e + source/probe launches"),
                     "steps_per_launch": steps_per_launch,
                     "launch_ms": round(launch_ms, 5),
                     "algorithmic_bytes_per_step": bytes_step,
                     "algorithmic_bytes_per_launch": bytes_launch,
                     "dram_gbs": (round(traffic / (launch_ms * 1e-3) / 1e9, 1) if traffic else None)},
        "gpu_launches": K * ((launches if w.get("dim", 2) == 2 else 3 * w["steps"]) + 3),
        "clocks": clk.summary(),
    }
    if e2e:
        line["e2e"] = e2e
    if cpu:
        line["cpu_baseline"] = cpu
    if grad4:
        line["config4_gradient"] = grad4
    if pack3:
        line["config3_packed"] = pack3
    if fwd5:
        line["config5_forward"] = fwd5
    print(json.dumps(line), flush=True)


class _HostMaps:
    """A phantom's host maps, evaluated once before timing: the caller's input
    arrays (generating the phantom is not part of the measured path)."""

    def __init__(self, ph):
        three = hasattr(ph, "get_eps_map_3d")
        self.eps_r, self.sigma = ph.get_eps_map_3d() if three else ph.get_eps_map()
        self.dispersion = ph.get_dispersion()
        if three:
            self.get_eps_map_3d = self.get_eps_map

    def get_eps_map(self, frequency=None):
        return self.eps_r, self.sigma

    def get_dispersion(self):
        return self.dispersion


def apply_temporal_block(solver, w, steps):
    """Steps per launch for a 2D workload's solver, set explicitly whatever it
    is (the solver's own default is two); 3D workloads run one step per
    launch.  Returns the steps per launch in use."""
    if w.get("dim", 2) != 2:
        return 1
    solver.set_temporal_block(steps)
    return steps


def run_e2e(w, phantoms, pos, freqs, device, tblock=1, rows=0):
    """Public-API path per sample: host phantom maps -> set_phantom ->
    update_materials (H2D of the FP64 maps) -> run() (D2H of every series) ->
    s_matrix() (D2H) -> DAS image (D2H)."""
    import torch
    from ceep_b200 import BatchedFDTD2D, BatchedFDTD3D
    from ceep_b200.spectral import das_image
    three = w.get("dim", 2) == 3
    if three:
        solver = BatchedFDTD3D(w["nx"], w["ny"], w["nz"], w["dx"], w["steps"], w["cpml"], pos, pos, 2e9,
                               frequencies=freqs, device=str(device))
    else:
        solver = BatchedFDTD2D(w["nx"], w["ny"], w["dx"], w["steps"], w["cpml"], pos, pos, 2e9,
                               frequencies=freqs, device=str(device), temporal_block=tblock,
                               rows_per_block=rows)   # the tile height the device-timed run tuned
    half = 0.07 if three else 0.09
    phantoms = [None if ph is None else _HostMaps(ph) for ph in phantoms]

    def sample(ph):
        solver.reset()
        if ph is not None:
            solver.set_phantom(ph)
        solver.update_materials()
        solver.run()
        S = solver.s_matrix()
        img = das_image(torch.as_tensor(S, dtype=torch.complex64, device=device), freqs,
                        np.asarray([p[:2] for p in pos], float) * w["dx"], w["das"], w["das"],
                        w["nx"] // 2 * w["dx"] - half, w["ny"] // 2 * w["dx"] - half, 2 * half / w["das"],
                        299_792_458.0).cpu().numpy()
        return S, img

    if phantoms[0] is not None:
        solver.set_phantom(phantoms[0])
    solver.run()  # builds and captures the graph once
    sample(phantoms[0])  # one untimed pass of the whole path (first use of every kernel module)
    torch.cuda.synchronize()
    h2d = d2h = 0
    times = []
    for ph in phantoms:
        t0 = time.perf_counter()
        S, img = sample(ph)
        times.append(time.perf_counter() - t0)
        # FP64 maps: eps_r, sigma and 2 per Debye / 3 per Lorentz pole; S for the image
        h2d = _cells(w) * 8 * (2 + 2 * len(solver._debye) + 3 * len(solver._lorentz)) + S.size * 8
        d2h = solver.probe_data.numel() * 4 + S.size * 8 + img.size * 4
    cell_steps = _cells(w) * w["steps"] * w["ntx"]
    name = "BatchedFDTD3D" if three else "BatchedFDTD2D"
    # median sample: the host-timed path sees occasional stalls of the Python host
    return {"value": round(cell_steps / float(np.median(times)) / 1e9, 3), "unit": "GCell-steps/s",
            "samples": len(times), "sample_ms": [round(t * 1e3, 2) for t in times],
            "h2d_bytes_per_step": int(h2d), "d2h_bytes_per_step": int(d2h),
            "path": f"{name}.set_phantom/run/s_matrix + DAS, host arrays in and out"}


def _oracle_worker_init(w, tx_list, seed):
    """One oracle over the TX in ``tx_list`` of workload ``w``: the 2D disk
    (config 1), the 2D Debye head (config 2, or a config-3 pack case when
    ``w`` names its phantom), or the 3D Debye head (config 5)."""
    global _ORACLE
    from ceep_b200.phantoms import HeadPhantom2D, HeadPhantom3D, ring_positions
    if w.get("dim", 2) == 3:
        from oracle.fdtd3d import Fdtd3DOracle
        pos = [(x, y, w["nz"] // 2) for x, y in ring_positions(w["ntx"], (w["nx"] // 2, w["ny"] // 2), w["ring"])]
        sc = min(w["nx"], w["ny"], w["nz"]) / 192.0
        ph = HeadPhantom3D(w["nx"], w["ny"], w["nz"], w["dx"], seed=seed,
                           semi_axes=(0.070 * sc, 0.056 * sc, 0.060 * sc))
        eps, sig = ph.get_eps_map_3d()
        _ORACLE = Fdtd3DOracle(w["nx"], w["ny"], w["nz"], w["dx"], w["steps"], w["cpml"], [pos[i] for i in tx_list],
                               pos, 2e9, eps_r=eps, sigma_e=sig, dispersion=ph.get_dispersion())
        return
    from oracle.fdtd2d import Fdtd2DOracle
    pos = ring_positions(w["ntx"], (w["nx"] // 2, w["ny"] // 2), w["ring"])
    src = [pos[i] for i in tx_list]
    if "phantom" in w:
        ph = _case_phantom(w)
        eps, sig = ph.get_eps_map()
        disp = ph.get_dispersion()
    elif w["debye"]:
        ph = HeadPhantom2D(w["nx"], w["ny"], w["dx"], seed=seed)
        eps, sig = ph.get_eps_map()
        disp = ph.get_dispersion()
    else:
        x, y = np.meshgrid(np.arange(w["nx"]), np.arange(w["ny"]), indexing="ij")
        m = (x - w["nx"] // 2) ** 2 + (y - w["ny"] // 2) ** 2 <= 40 ** 2
        eps, sig, disp = np.where(m, 40.0, 1.0), np.where(m, 0.5, 0.0), None
    _ORACLE = Fdtd2DOracle(w["nx"], w["ny"], w["dx"], w["steps"], w["cpml"], src, pos, 2e9,
                           eps_r=eps, sigma_e=sig, dispersion=disp)


def _oracle_worker_run(nsteps):
    t0 = time.perf_counter()
    for _ in range(nsteps):
        if _ORACLE.step_index >= _ORACLE.total_steps:
            _ORACLE.step_index = 0
        _ORACLE.step()
    return time.perf_counter() - t0


def cpu_baseline(w, sample_steps=12):
    """Oracle port, one process (NumPy elementwise is single-threaded), on a
    bounded number of time steps of the same workload."""
    _oracle_worker_init(w, list(range(w["ntx"])), 1000)
    dt = _oracle_worker_run(sample_steps)
    v = _cells(w) * w["ntx"] * sample_steps / dt / 1e9
    return {"value": round(v, 6), "unit": "GCell-steps/s", "cores": 1, "kind": "port",
            "sample": f"{sample_steps} of {w['steps']} time steps, all {w['ntx']} TX, FP64 NumPy oracle, "
                      f"{dt:.1f} s"}


def _cells(w):
    return w["nx"] * w["ny"] * w.get("nz", 1)


def _time_oracle_pools(cases, ncpu, warmup, steps, per_step):
    """Spread the TX of every case in ``cases`` (workload dicts) over spawn
    workers, one oracle per worker; time ``steps`` bench steps of ``per_step``
    time steps each after ``warmup`` one-step rounds.  Returns (seconds per
    bench step, worker count)."""
    import multiprocessing as mp
    ctx = mp.get_context("spawn")
    share = max(1, ncpu // len(cases))
    jobs = []
    for w in cases:
        nproc = max(1, min(share, w["ntx"]))
        jobs += [(w, list(range(w["ntx"]))[i::nproc]) for i in range(nproc)]
    pools = [ctx.Pool(1, initializer=_oracle_worker_init, initargs=(w, g, w.get("seed", 1000))) for w, g in jobs]
    try:
        for _ in range(warmup):
            [r.get() for r in [p.apply_async(_oracle_worker_run, (1,)) for p in pools]]
        times = []
        for _ in range(steps):
            t0 = time.perf_counter()
            [r.get() for r in [p.apply_async(_oracle_worker_run, (per_step,)) for p in pools]]
            times.append(time.perf_counter() - t0)
    finally:
        for p in pools:
            p.close()
            p.join()
    return times, len(pools)


def _reference_line(args, workload, value, ms, cores, sample, config, metric="batched FDTD GCell-steps/s",
                    dtype="f64"):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    line = {"impl": "reference", "metric": metric, "value": round(value, 6), "unit": "GCell-steps/s",
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(ms, 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": "synthetic (seeded phantoms)", "config": dict(workload=workload, **config),
            "cpu_baseline": {"value": round(value, 6), "unit": "GCell-steps/s", "cores": cores, "kind": "port",
                             "sample": sample},
            "e2e": {"value": round(value, 6), "unit": "GCell-steps/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_reference(args, w):
    """Reference arm: the oracle port on all host cores (TX spread over spawn
    workers), a bounded number of time steps per bench step."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    ncpu = os.cpu_count() or 1
    per_step = args.cpu_steps if w.get("dim", 2) == 2 else max(1, args.cpu_steps // 6)
    times, nproc = _time_oracle_pools([w], ncpu, args.warmup, args.steps, per_step)
    value = len(times) * _cells(w) * w["ntx"] * per_step / sum(times) / 1e9
    cfg = {k: w[k] for k in ("nx", "ny", "nz") if k in w}
    cfg.update(tx=w["ntx"], time_steps_per_bench_step=per_step)
    _reference_line(args, args.workload, value, 1e3 * sum(times) / len(times), nproc,
                    f"{per_step} time steps x {w['ntx']} TX per bench step, {nproc} spawn workers over TX, "
                    f"{ncpu} host cores", cfg)


def run_pack_reference(args):
    """Reference arm of the packed uneven batch: the 2D oracle on a sample of
    the config-3 phantoms (every TX of each, spread over spawn workers), a
    bounded number of time steps per bench step."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    ncpu = os.cpu_count() or 1
    cases = _pack_cases(args.pack_count)
    sample = cases[:: max(1, len(cases) // 4)][:4]
    per_step = args.cpu_steps
    times, nproc = _time_oracle_pools(sample, ncpu, args.warmup, args.steps, per_step)
    cs = sum(_cells(c) * c["ntx"] for c in sample) * per_step
    value = len(times) * cs / sum(times) / 1e9
    _reference_line(args, "pack256", value, 1e3 * sum(times) / len(times), nproc,
                    f"{len(sample)} of {args.pack_count} phantoms ({', '.join(f'{c['nx']}x{c['ny']}' for c in sample)}),"
                    f" all TX, {per_step} time steps each per bench step, {nproc} spawn workers",
                    {"phantoms": args.pack_count, "sampled": len(sample), "time_steps_per_bench_step": per_step},
                    metric="packed uneven batch GCell-steps/s")


def _single_case(nx):
    """The non-batched workload: TMz, nx x nx, 1 mm, CFS-CPML 20, a Gaussian Ez
    source at the centre, eight probes on a circle, a lossy dielectric disk of
    radius nx/5 (eps_r 4, sigma 0.2 S/m)."""
    from ceep_b200 import fdtd2d as F
    T, n = 1000, 20
    cfg = F.SimulationConfig(grid=F.GridConfig(nx=nx, ny=nx, dx=1e-3, dy=1e-3), mode=F.SimulationMode.TMZ,
                             total_steps=T)
    src = [F.GaussianSource(x=nx // 2, y=nx // 2, frequency_max=20e9)]
    prb = [(nx // 2 + int(0.3 * nx * np.cos(a)), nx // 2 + int(0.3 * nx * np.sin(a)))
           for a in np.linspace(0, 2 * np.pi, 8, endpoint=False)]
    return cfg, src, prb, n, T


def _single_oracle(nx):
    """The oracle of ``_single_case``: coefficients from the disk map in FP64
    (the update coefficients of grid.py:157-195)."""
    from oracle.fdtd2d_single import EPS_0, MU_0, Single2DOracle
    cfg, src, prb, n, T = _single_case(nx)
    dt = cfg.dt
    x, y = np.meshgrid(np.arange(nx), np.arange(nx), indexing="ij")
    m = (x - nx // 2) ** 2 + (y - nx // 2) ** 2 <= (nx // 5) ** 2
    eps = np.where(m, 4.0, 1.0) * EPS_0
    se = np.where(m, 0.2, 0.0) * dt / (2.0 * eps)
    mu = MU_0
    ca, cb = (1.0 - se) / (1.0 + se), (dt / eps) / (1.0 + se)
    da, db = np.ones((nx, nx)), np.full((nx, nx), dt / mu)
    wave = np.array([src[0].value_at(k, dt) for k in range(T)])
    return Single2DOracle(nx, nx, 1e-3, 1e-3, dt, "TMZ", ca, cb, da, db, [(nx // 2, nx // 2, "Ez", wave)],
                          [("cpml", n, 4, 2.0, 0.05, 1.0)], prb), T


def run_single_reference(args):
    """Reference arm of the non-batched solver: the oracle (one NumPy process,
    as the reference's own NumPy backend runs) for a bounded number of time
    steps per bench step."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    nx = 1024 if args.small else 4096
    o, T = _single_oracle(nx)
    per_step = 2
    o.run(args.warmup)
    times = []
    for _ in range(args.steps):
        if o.n + per_step > T:
            o.n = 0
        t0 = time.perf_counter()
        o.run(per_step)
        times.append(time.perf_counter() - t0)
    value = len(times) * nx * nx * per_step / sum(times) / 1e9
    _reference_line(args, "single4096" if not args.small else "single1024", value, 1e3 * sum(times) / len(times), 1,
                    f"{per_step} of {T} time steps per bench step, FP64 NumPy oracle, one process",
                    {"nx": nx, "ny": nx, "mode": "TMz", "cpml": 20, "time_steps_per_bench_step": per_step},
                    metric="FDTD2D (non-batched) GCell-steps/s")


def run_adjoint_reference(args):
    if int(os.environ.get("RANK", "0")) != 0:
        return
    print(json.dumps({"impl": "reference", "workload": args.workload,
                      "unavailable": "the reference computes no gradient of its solvers (no adjoint path)"}),
          flush=True)


def adjoint400_ratios(Ks=(1, 25, 50, 100), keep_budget=16 << 30, reps=2, split=True):
    """Config 4: cost of a full S-misfit gradient (forward with checkpoints +
    segment recompute + adjoint) relative to one plain forward, for the
    checkpoint intervals `Ks` (and, with `keep_budget`, again with trailing
    segments kept within that many bytes).  400x400, 0.5 mm, 1000 steps,
    CPML 15, 16 TX/RX, 101 frequencies, one-pole Debye head phantom (scaled
    to the grid); target S from the phantom with its disk, parameters from the
    phantom without it.  Returns (forward ms, ratios, kept ratios, kept info,
    the K = 1 split)."""
    import torch
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.adjoint import Adjoint2D, probes_with_grad, s_parameter_loss
    from ceep_b200.phantoms import HeadPhantom2D, ring_positions
    dev = torch.device("cuda", 0)
    nx = ny = 400
    T, n = 1000, 15
    pos = ring_positions(16, (nx // 2, ny // 2), 130)
    freqs = np.linspace(0.5e9, 3.5e9, 101)
    kw = dict(nx=nx, ny=ny, dx=0.5e-3, seed=7, semi_axes=(0.060, 0.047))
    with_disk = HeadPhantom2D(p_disk=1.0, **kw)
    no_disk = HeadPhantom2D(p_disk=0.0, **kw)
    # the target
    s = BatchedFDTD2D(nx, ny, 0.5e-3, T, n, pos, pos, 2e9, frequencies=freqs, device=str(dev))
    s.set_phantom(with_disk)
    s.run()
    target = torch.as_tensor(s.s_matrix(), device=dev)
    eps, sig = no_disk.get_eps_map()
    de, tau = no_disk.get_dispersion()["debye"][0]
    f64 = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)
    # one plain forward (graph-replayed), the unit of cost
    s2 = BatchedFDTD2D(nx, ny, 0.5e-3, T, n, pos, pos, 2e9, device=str(dev))
    s2.set_phantom(no_disk)
    s2._build()
    stream = torch.cuda.current_stream(dev)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    def fwd():
        s2.reset()
        s2.advance(0, T, stream=stream)
    t_fwd = timed(fwd, 3)
    ratios, kept_ratios, kept_info, split_ms = {}, {}, {}, None
    cases = [(K, 0) for K in Ks] + ([(K, keep_budget) for K in Ks if K > 1] if keep_budget else [])
    for K, keep in cases:
        sk = BatchedFDTD2D(nx, ny, 0.5e-3, T, n, pos, pos, 2e9, device=str(dev))
        sk.set_phantom(no_disk)
        adj = Adjoint2D(sk, checkpoint_every=K, keep_bytes=keep)
        e, g = f64(eps).requires_grad_(True), f64(sig).requires_grad_(True)
        d = f64(de).requires_grad_(True)

        def grad_step():
            e.grad = g.grad = d.grad = None
            loss, _ = s_parameter_loss(probes_with_grad(e, g, adj, d, f64(tau)).double(), sk.dt, freqs, target)
            loss.backward()
        r = timed(grad_step, reps) / t_fwd
        if keep:
            kept_ratios[K] = r
            nseg = -(-T // K)
            kept_info[K] = f"{adj.kept_segments(nseg)} of {nseg} segments kept, " \
                           f"{adj.kept_segments(nseg) * adj.segment_bytes() / 2 ** 30:.2f} GiB"
            del adj, sk
            torch.cuda.empty_cache()
            continue
        ratios[K] = r
        if K == 1 and split:
            # split of one gradient: the forward that saves Ez/J of every step,
            # and the backward (adjoint steps + chain rule)
            adj.set_parameters(e.detach(), g.detach(), d.detach(), f64(tau))
            gprobe = torch.randn((len(pos), len(pos), T), dtype=torch.float32, device=dev)
            t_f = timed(adj.forward, 2)
            t_fb = timed(lambda: (adj.forward(), adj.backward(gprobe)), 2)
            split_ms = {"forward_save_ms": t_f, "backward_ms": t_fb - t_f}
        del adj, sk
        torch.cuda.empty_cache()
    return t_fwd, ratios, kept_ratios, kept_info, split_ms


def run_adjoint_bench(args):
    """Config 4 on its own line: adjoint400_ratios at K = 1, 25, 50, 100 with
    and without a 16 GiB keep budget."""
    keep_budget = 16 << 30
    t_fwd, ratios, kept_ratios, kept_info, split = adjoint400_ratios(keep_budget=keep_budget)
    line = {"metric": "adjoint gradient cost vs forward", "value": round(ratios[50], 3), "unit": "x forward",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f32", "data": "synthetic (seeded phantom)",
            "config": {"workload": "adjoint400", "nx": 400, "ny": 400, "time_steps": 1000, "tx": 16, "cpml": 15,
                       "debye_poles": 1, "dft_freqs": 101, "loss": "sum |S - S*|^2",
                       "grad": "eps_r, sigma, debye delta_eps"},
            "forward_ms": round(t_fwd, 3), "ratio_by_checkpoint_interval": {str(k): round(v, 3) for k, v in ratios.items()},
            "every_step_kept": {k: round(v, 3) for k, v in split.items()},
            "ratio_with_keep_budget": {str(k): round(v, 3) for k, v in kept_ratios.items()},
            "keep_budget": {"bytes": keep_budget, **{str(k): v for k, v in kept_info.items()}}}
    print(json.dumps(line), flush=True)


def run_adjoint3d_bench(args):
    """Config 5's gradient: 192^3, 1 mm, 1000 steps, CPML 10, 8 z-directed
    TX/RX on a mid-plane ring, 101 frequencies, Debye ellipsoid-shell head;
    target S from the head with its inclusion, parameters from the same head
    without it; d(S-misfit)/d(eps_r, sigma, delta_eps) through the
    checkpointed 3D adjoint, timed against one plain forward."""
    import torch
    from ceep_b200 import BatchedFDTD3D
    from ceep_b200.adjoint import s_parameter_loss
    from ceep_b200.adjoint3d import Adjoint3D, probes_with_grad_3d
    from ceep_b200.phantoms import HeadPhantom3D, ring_positions
    dev = torch.device("cuda", 0)
    w = WORKLOADS["head192"]
    nx, ny, nz, T, n = w["nx"], w["ny"], w["nz"], w["steps"], w["cpml"]
    if args.small:
        nx = ny = nz = 96
        T = 300
    c = nx // 2
    pos = [(x, y, nz // 2) for x, y in ring_positions(w["ntx"], (c, ny // 2), w["ring"] * nx // 192)]
    freqs = np.linspace(0.5e9, 3.5e9, w["nfreq"])
    sc = nx / 192.0
    kw = dict(nx=nx, ny=ny, nz=nz, dx=w["dx"], seed=7, semi_axes=(0.070 * sc, 0.056 * sc, 0.060 * sc))
    truth, guess = HeadPhantom3D(**kw), HeadPhantom3D(with_inclusion=False, **kw)
    mk = lambda: BatchedFDTD3D(nx, ny, nz, w["dx"], T, n, pos, pos, 2e9, frequencies=freqs, device=str(dev))
    s = mk()
    s.set_phantom(truth)
    s.run()
    target = torch.as_tensor(s.s_matrix(), device=dev)
    del s
    eps, sig = guess.get_eps_map_3d()
    de, tau = guess.get_dispersion()["debye"][0]
    f64 = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)
    stream = torch.cuda.current_stream(dev)

    def timed(fn, reps):
        fn()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        for _ in range(reps):
            fn()
        b.record(stream)
        torch.cuda.synchronize()
        return a.elapsed_time(b) / reps

    s2 = mk()
    s2.set_phantom(guess)
    s2._build()

    def fwd():
        s2.reset()
        s2.advance(0, T, stream=stream)
    t_fwd = timed(fwd, 3)
    del s2
    torch.cuda.empty_cache()
    ratios, mem, split = {}, {}, {}
    kept_ratios, kept_info = {}, {}
    keep_budget = 64 << 30
    for K, keep in ((25, 0), (50, 0), (100, 0), (25, keep_budget), (50, keep_budget)):
        torch.cuda.reset_peak_memory_stats(dev)
        sk = mk()
        sk.set_phantom(guess)
        adj = Adjoint3D(sk, checkpoint_every=K, keep_bytes=keep)
        e, g, d = f64(eps).requires_grad_(True), f64(sig).requires_grad_(True), f64(de).requires_grad_(True)

        def grad_step():
            e.grad = g.grad = d.grad = None
            p = probes_with_grad_3d(e, g, adj, d, f64(tau))
            loss, _ = s_parameter_loss(p.double(), sk.dt, freqs, target)
            loss.backward()
        r = timed(grad_step, 1) / t_fwd
        if keep:
            nseg = -(-T // K)
            kept_ratios[K] = r
            kept_info[K] = (f"{adj.kept_segments(nseg)} of {nseg} segments kept, peak "
                            f"{torch.cuda.max_memory_allocated(dev) / 2 ** 30:.1f} GiB")
            del adj, sk, e, g, d
            torch.cuda.empty_cache()
            continue
        ratios[K] = r
        mem[K] = torch.cuda.max_memory_allocated(dev) / 2 ** 30
        if K == 50:
            gprobe = torch.randn((len(pos), len(pos), T), dtype=torch.float32, device=dev)
            adj.set_parameters(e.detach(), g.detach(), d.detach(), f64(tau))
            t_f = timed(adj.forward, 1)
            t_fb = timed(lambda: (adj.forward(), adj.backward(gprobe)), 1)
            split = {"forward_ms": t_f, "backward_ms": t_fb - t_f}
        del adj, sk, e, g, d
        torch.cuda.empty_cache()
    line = {"metric": "adjoint gradient cost vs forward", "value": round(ratios[50], 3), "unit": "x forward",
            "higher_is_better": False, "n_gpus": 1, "dtype": "f32", "data": "synthetic (seeded phantom)",
            "config": {"workload": "adjoint192", "nx": nx, "ny": ny, "nz": nz, "time_steps": T,
                       "tx": len(pos), "cpml": n, "debye_poles": 1, "dft_freqs": len(freqs),
                       "loss": "sum |S - S*|^2", "grad": "eps_r, sigma, debye delta_eps"},
            "forward_ms": round(t_fwd, 3),
            "ratio_by_checkpoint_interval": {str(k): round(v, 3) for k, v in ratios.items()},
            "peak_device_gib_by_checkpoint_interval": {str(k): round(v, 1) for k, v in mem.items()},
            "checkpoint50_split_ms": {k: round(v, 3) for k, v in split.items()},
            "ratio_with_keep_budget": {str(k): round(v, 3) for k, v in kept_ratios.items()},
            "keep_budget": {"bytes": keep_budget, **{str(k): v for k, v in kept_info.items()}}}
    print(json.dumps(line), flush=True)


def single_bytes_per_cell_step(mode, n, nx, ny):
    """Unblocked compulsory bytes of one step of the non-batched solver: the
    three fields read and written (24 B per cell) and the four update
    coefficients (16 B per cell), plus psi read+write (8 B) per CPML strip
    cell and field: 2 for TMz cells on the x strips (Hy, Ez) and the y strips
    (Hx, Ez), same count for TEz."""
    strip_x = 2 * n * ny
    strip_y = 2 * n * nx
    return 40 * nx * ny + 2 * 8 * (strip_x + strip_y)


def run_single_bench(args):
    """The non-batched FDTD2D (fdtd_2d.py) on a grid well above L2: TMz,
    4096 x 4096, 1 mm, CFS-CPML 20 cells, a Gaussian Ez source at the centre,
    eight probes, 1000 steps per bench step; GCell-steps/s (cells x steps)."""
    import torch
    from ceep_b200 import fdtd2d as F
    dev = torch.device("cuda", 0)
    nx = ny = 1024 if args.small else 4096
    cfg, src, prb, n, T = _single_case(nx)
    s = F.FDTD2D(cfg, sources=src, boundaries=[F.CPML(thickness=n)], probe_points=prb)
    s.grid.set_material_circle(nx // 2, ny // 2, nx // 5, eps_r=4.0, sigma_e=0.2)
    stream = torch.cuda.current_stream(dev)
    flush = torch.empty(64 * 2 ** 20, dtype=torch.float32, device=dev)   # 256 MB

    def one():
        s.reset()
        s.advance(T, stream=stream)
    for _ in range(args.warmup):
        one()
    torch.cuda.synchronize()
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    with ClockSampler(0) as clk:
        for a, b in ev:
            flush.zero_()
            a.record(stream)
            one()
            b.record(stream)
        torch.cuda.synchronize()
    ms = [a.elapsed_time(b) for a, b in ev]
    total = float(np.sum(ms))
    value = len(ms) * nx * ny * T / (total * 1e-3) / 1e9
    step_ms = float(np.median(ms)) / T
    peak, src_peak = hbm_peak()
    bytes_step = single_bytes_per_cell_step("TMZ", n, nx, ny)
    achieved = bytes_step / (step_ms * 1e-3) / 1e9
    # e2e through the public API: maps and sources in from the host, run(),
    # probe series back as host lists
    # (median of three fresh solvers: the host part varies from run to run)
    host_eps = s.grid.eps_r.copy()
    e2e_runs = []
    for _ in range(3):
        t0 = torch.cuda.Event(enable_timing=True)
        t1 = torch.cuda.Event(enable_timing=True)
        t0.record(stream)
        s2 = F.FDTD2D(cfg, sources=src, boundaries=[F.CPML(thickness=n)], probe_points=prb)
        s2.grid.eps_r[:] = host_eps
        s2.grid.eps_inf[:] = host_eps
        s2.grid.sigma_e[:] = s.grid.sigma_e
        s2.grid._precompute_coefficients()
        s2.run()
        t1.record(stream)
        torch.cuda.synchronize()
        e2e_runs.append(t0.elapsed_time(t1))
        del s2
    e2e_ms = float(np.median(e2e_runs))
    cpu = None
    if not args.no_cpu:
        o, _ = _single_oracle(nx)
        k = 6
        t = time.perf_counter()
        o.run(k)
        el = time.perf_counter() - t
        cpu = {"value": round(nx * ny * k / el / 1e9, 5), "unit": "GCell-steps/s", "cores": 1, "kind": "port",
               "sample": f"{k} of {T} time steps, FP64 NumPy oracle, {el:.1f} s"}
    line = {"metric": "FDTD2D (non-batched) GCell-steps/s", "value": round(value, 3), "unit": "GCell-steps/s",
            "n_gpus": 1, "steps": len(ms), "warmup": args.warmup, "ms_per_step": round(total / len(ms), 3),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (dielectric disk)",
            "config": {"workload": "single4096" if not args.small else "single1024", "nx": nx, "ny": ny,
                       "mode": "TMz", "time_steps": T, "cpml": n, "boundary": "CFS-CPML",
                       "l2": "256 MB flush before every bench step; state 335 MB > L2"},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 3), "traffic": None, "peak_source": src_peak,
                         "kernel": "single2d_step_kernel interior + frame launches (+ record) per step",
                         "algorithmic_bytes_per_step": bytes_step, "step_ms": round(step_ms, 5)},
            "e2e": {"value": round(nx * ny * T / (e2e_ms * 1e-3) / 1e9, 3), "unit": "GCell-steps/s",
                    "h2d_bytes_per_step": 8 * 4 * nx * ny, "d2h_bytes_per_step": 4 * len(prb) * T,
                    "path": "FDTD2D(...) + set materials + run(), probe lists back on the host; the four FP64 "
                            "material maps go up, the coefficients are formed on the device; median of 3 fresh "
                            "solvers"},
            "gpu_launches": len(ms) * 3 * T,
            "clocks": clk.summary()}
    if cpu:
        line["cpu_baseline"] = cpu
    print(json.dumps(line), flush=True)


def _pack_cases(count, seed=2024):
    """Config-3 phantoms as host-side specs: nx, ny in {256..768 step 32},
    steps in [600, 1200], 8-16 TX on a ring, one third with a two-pole
    Lorentz model instead of Debye."""
    rng = np.random.default_rng(seed)
    sizes = np.arange(256, 769, 32)
    out = []
    for k in range(count):
        nx, ny = int(rng.choice(sizes)), int(rng.choice(sizes))
        steps, ntx = int(rng.integers(600, 1201)), int(rng.integers(8, 17))
        scale = min(nx, ny) / 600.0
        out.append(dict(nx=nx, ny=ny, dx=0.5e-3, steps=steps, cpml=15, ntx=ntx, ring=0.36 * min(nx, ny),
                        debye=True, phantom="lorentz" if k % 3 == 2 else "head",
                        semi_axes=(0.09 * scale, 0.07 * scale), seed=seed + k))
    return out


def _case_phantom(c):
    from ceep_b200.phantoms import HeadPhantom2D, LorentzHeadPhantom2D
    cls = LorentzHeadPhantom2D if c["phantom"] == "lorentz" else HeadPhantom2D
    return cls(nx=c["nx"], ny=c["ny"], dx=c["dx"], seed=c["seed"], semi_axes=c["semi_axes"])


def _pack_solvers(count, device, seed=2024):
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.phantoms import ring_positions
    out = []
    for c in _pack_cases(count, seed):
        pos = ring_positions(c["ntx"], (c["nx"] // 2, c["ny"] // 2), c["ring"])
        s = BatchedFDTD2D(c["nx"], c["ny"], c["dx"], c["steps"], c["cpml"], pos, pos, 2e9, device=str(device))
        s.set_phantom(_case_phantom(c))
        out.append(s)
    return out


def _pack_launch_count(solvers, tblock):
    """Kernel launches of one packed run: per class (lane width x ADE shape)
    one launch per step (tblock 1), or per step pair one two-step launch while
    any phantom has two steps left plus one one-step launch where a phantom
    takes its odd last step alone (tblock 2)."""
    classes = {}
    for s in solvers:
        classes.setdefault((s._gwidth, len(s._debye), len(s._lorentz)), []).append(s.total_steps)
    n = 0
    for steps in classes.values():
        top = max(steps)
        if tblock == 1:
            n += top
        else:
            for t in range((top + 1) // 2):
                n += any(x >= 2 * t + 2 for x in steps) + any(x == 2 * t + 1 for x in steps)
    return n


def _graph_launch_gap_us(dev, stream, n=2000):
    """Device time per launch of a CUDA graph of `n` launches of a one-element
    kernel: an upper bound of what a graph of launches loses between kernels
    (the cost a single persistent launch would save)."""
    import torch
    x = torch.zeros(1, device=dev)
    x.add_(1.0)
    torch.cuda.synchronize()
    g = torch.cuda.CUDAGraph()
    with torch.cuda.graph(g):
        for _ in range(n):
            x.add_(1.0)
    g.replay()
    torch.cuda.synchronize()
    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    a.record(stream)
    g.replay()
    b.record(stream)
    torch.cuda.synchronize()
    return a.elapsed_time(b) * 1e3 / n


def head192_forward_figure():
    """Config 5's forward on its own (the 3D Debye head, 192^3 x 8 TX x 1000
    steps): one graph-replayed time loop, L2 flushed before it, against the
    3D formula's compulsory bytes."""
    import torch
    dev = torch.device("cuda", 0)
    w = WORKLOADS["head192"]
    solver, _, _, phantoms, _ = build_inputs_3d(w, 1, dev)
    stream = torch.cuda.current_stream(dev)
    solver.advance(0, w["steps"], stream=stream)  # capture + warm
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    times = []
    for _ in range(2):
        flush.zero_()
        solver.reset()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        solver.advance(0, w["steps"], stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b) * 1e-3)
    t = float(min(times))
    n_debye = len(phantoms[0].get_dispersion()["debye"])
    peak, _ = hbm_peak()
    bytes_step = algorithmic_bytes_per_step_3d(w, n_debye)
    out = {"workload": "head192 forward (192^3, 1 mm, 1000 steps, 8 TX, Debye head)",
           "value": round(w["nx"] * w["ny"] * w["nz"] * w["steps"] * w["ntx"] / t / 1e9, 3),
           "unit": "GCell-steps/s", "ms_per_run": round(t * 1e3, 2),
           "roofline_frac": round(bytes_step * w["steps"] / t / 1e9 / peak, 3)}
    del solver, flush
    torch.cuda.empty_cache()
    return out


def pack_measure(count, pack_sample, steps):
    """Config 3: one packed, graph-replayed run of `count` seeded phantoms
    (autotuned), its per-phantom baselines on a sample, and its roofline.
    Returns the figures run_pack_bench prints."""
    import torch
    from ceep_b200.packed import PackedBatch2D
    dev = torch.device("cuda", 0)
    stream = torch.cuda.current_stream(dev)
    # baseline: per-phantom run() on a sample (fresh solver = what a caller does)
    sample = _pack_solvers(count, dev)[:: max(1, count // pack_sample)]
    t_fresh = t_replay = cs_sample = 0.0
    for s in sample:
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        s.run()
        torch.cuda.synchronize()
        t_fresh += time.perf_counter() - t0
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.reset()
        a.record(stream)
        s.advance(0, s.total_steps, stream=stream)
        b.record(stream)
        torch.cuda.synchronize()
        t_replay += a.elapsed_time(b) / 1e3
        cs_sample += s.nx * s.ny * s.total_steps * s.batch
    del sample
    torch.cuda.empty_cache()
    solvers = _pack_solvers(count, dev)
    pk = PackedBatch2D(solvers)
    timings = pk.autotune(candidates=(12, 16, 24, 32), probe_steps=30)
    pk.reset()
    pk.advance(0, pk.max_steps, stream)          # graph capture of the full run
    torch.cuda.synchronize()
    times = []
    for _ in range(steps):
        pk.reset()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        pk.advance(0, pk.max_steps, stream)
        b.record(stream)
        torch.cuda.synchronize()
        times.append(a.elapsed_time(b) / 1e3)
    for s in solvers:
        s.check_status()
    value = pk.cell_steps / float(np.median(times)) / 1e9
    launches = _pack_launch_count(solvers, pk.temporal_block)
    gap_us = _graph_launch_gap_us(dev, stream)
    # roofline of the whole packed run: compulsory bytes of every phantom's
    # steps (real TX counts, not the padded lanes) over the run's time
    alg = sum(algorithmic_bytes_per_step_2d({"nx": s.nx, "ny": s.ny, "cpml": s.cpml_n, "ntx": s.batch},
                                            len(s._debye), len(s._lorentz)) * s.total_steps for s in solvers)
    peak, peak_src = hbm_peak()
    achieved = alg / float(np.median(times)) / 1e9
    base_fresh = cs_sample / t_fresh / 1e9
    base_replay = cs_sample / t_replay / 1e9
    out = {"value": value, "pk": pk, "timings": timings, "alg": alg, "peak": peak, "peak_src": peak_src,
           "achieved": achieved, "launches": launches, "gap_us": gap_us, "run_s": float(np.median(times)),
           "base_fresh": base_fresh, "base_replay": base_replay,
           "baseline_sample": len(range(0, count, max(1, count // pack_sample)))}
    del solvers
    return out


def run_pack_bench(args):
    """Config 3: aggregate GCell-steps/s of one packed, graph-replayed run of
    all phantoms against per-phantom run() calls of the single-grid kernel."""
    m = pack_measure(args.pack_count, args.pack_sample, args.steps)
    pk, value, achieved, peak = m["pk"], m["value"], m["achieved"], m["peak"]
    line = {"metric": "packed uneven batch GCell-steps/s", "value": round(value, 3), "unit": "GCell-steps/s",
            "n_gpus": 1, "steps": args.steps, "higher_is_better": True, "dtype": "f32",
            "data": "synthetic (seeded phantoms)",
            "config": {"workload": "pack256", "phantoms": args.pack_count, "sizes": "256..768 step 32",
                       "time_steps": "600..1200", "tx": "8..16", "lorentz_fraction": "1/3", "cpml": 15,
                       "tile_rows": pk.rows, "cell_steps": pk.cell_steps},
            "roofline": {"bound": "hbm", "achieved": round(achieved, 1), "peak": peak, "unit": "GB/s",
                         "frac": round(achieved / peak, 3), "peak_source": m["peak_src"],
                         "algorithmic_bytes": int(m["alg"]), "kernel": ("fdtd2d_packed2_kernel, two steps per launch" if pk.temporal_block == 2 else "fdtd2d_packed_kernel") + " (whole run)", "temporal_block": pk.temporal_block,
                         "packing": ("concurrent class chains" if pk.packing else "interleaved") + f" ({pk.classes} classes)"},
            "autotune_ms_per_step": {str(k): round(v, 4) for k, v in m["timings"].items()},
            "graph_launches": m["launches"], "graph_launch_gap_us": round(m["gap_us"], 3),
            "launch_gap_share": round(m["launches"] * m["gap_us"] * 1e-6 / m["run_s"], 5),
            "per_phantom_run_gcells": round(m["base_fresh"], 3), "per_phantom_replay_gcells": round(m["base_replay"], 3),
            "speedup_vs_run": round(value / m["base_fresh"], 2), "speedup_vs_replay": round(value / m["base_replay"], 2),
            "baseline_sample": m["baseline_sample"]}
    print(json.dumps(line), flush=True)


def run_profile_adjoint(args):
    """One gradient (forward with one checkpoint segment + adjoint) of a
    400x400, 16-TX Debye case over --profile steps, launched without graphs."""
    import torch
    from ceep_b200 import BatchedFDTD2D
    from ceep_b200.adjoint import Adjoint2D, probes_with_grad
    from ceep_b200.phantoms import HeadPhantom2D, ring_positions
    dev = torch.device("cuda", 0)
    T = args.profile
    pos = ring_positions(16, (200, 200), 130)
    ph = HeadPhantom2D(nx=400, ny=400, dx=0.5e-3, seed=7, semi_axes=(0.060, 0.047))
    s = BatchedFDTD2D(400, 400, 0.5e-3, T, 15, pos, pos, 2e9, device=str(dev), use_graph=False)
    s.set_phantom(ph)
    eps, sig = ph.get_eps_map()
    de, tau = ph.get_dispersion()["debye"][0]
    f64 = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)
    e = f64(eps).requires_grad_(True)
    p = probes_with_grad(e, f64(sig), Adjoint2D(s, checkpoint_every=T), f64(de), f64(tau))
    (p.double() ** 2).sum().backward()
    torch.cuda.synchronize()
    print("profile run done", flush=True)


def run_profile_adjoint3d(args):
    """One gradient of a 192^3 (128^3 with --small), 8-TX Debye head over
    --profile steps (one checkpoint segment, so no recompute), launched
    without graphs."""
    import torch
    from ceep_b200 import BatchedFDTD3D
    from ceep_b200.adjoint3d import Adjoint3D, probes_with_grad_3d
    from ceep_b200.phantoms import HeadPhantom3D, ring_positions
    dev = torch.device("cuda", 0)
    T, nx = args.profile, (128 if args.small else 192)
    pos = [(x, y, nx // 2) for x, y in ring_positions(8, (nx // 2, nx // 2), 50 if args.small else 75)]
    sc = nx / 192.0
    ph = HeadPhantom3D(nx=nx, ny=nx, nz=nx, dx=1e-3, seed=7, semi_axes=(0.070 * sc, 0.056 * sc, 0.060 * sc))
    s = BatchedFDTD3D(nx, nx, nx, 1e-3, T, 10, pos, pos, 2e9, device=str(dev), use_graph=False)
    s.set_phantom(ph)
    eps, sig = ph.get_eps_map_3d()
    de, tau = ph.get_dispersion()["debye"][0]
    f64 = lambda a: torch.as_tensor(a, dtype=torch.float64, device=dev)
    e = f64(eps).requires_grad_(True)
    p = probes_with_grad_3d(e, f64(sig), Adjoint3D(s, checkpoint_every=T), f64(de), f64(tau))
    (p.double() ** 2).sum().backward()
    torch.cuda.synchronize()
    print("profile run done", flush=True)


def run_profile(args, w):
    """A few fused steps of one sample, launched without a graph, then the DFT
    and DAS once: the small command that ncu captures.  With --small the 3D
    workload shrinks to 128^3 (state ~0.6 GB) for multi-pass captures."""
    import torch
    device = torch.device("cuda", 0)
    if args.small and w.get("dim", 2) == 3:
        w = dict(w, nx=128, ny=128, nz=128, ring=50)
    solver, pos, freqs, _, mats = build_inputs(w, 1, device)
    solver.use_graph = False
    if args.rows and w.get("dim", 2) == 2:
        solver.set_rows_per_block(args.rows)
    apply_temporal_block(solver, w, args.temporal_block)
    solver.load_material_tensors(mats[0])
    stream = torch.cuda.current_stream(device)
    solver.advance(0, min(args.profile, w["steps"]), stream=stream)
    das_ws = torch.empty(1 << 20, dtype=torch.uint8, device=device)
    from ceep_b200.spectral import das_image, dft
    S = dft(solver.probe_data, freqs, solver.dt)
    das_image(S, freqs, np.asarray([p[:2] for p in pos], float) * w["dx"], w["das"], w["das"], 0.06, 0.06,
              0.18 / w["das"],
              299_792_458.0, True, workspace=das_ws)
    torch.cuda.synchronize()
    print("profile run done", flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="head600",
                    choices=list(WORKLOADS) + ["adjoint400", "adjoint192", "pack256", "single4096"])
    ap.add_argument("--pack-count", type=int, default=256)
    ap.add_argument("--pack-sample", type=int, default=32)
    ap.add_argument("--small", action="store_true", help="a smaller grid (--profile of the 3D gradient: 128^3; "
                                                         "single4096: 1024^2)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--temporal-block", type=int, default=2, choices=(1, 2),
                    help="2D steps per kernel launch (2 = temporal block of two)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-autotune", action="store_true", help="2D: keep the automatic tile height")
    ap.add_argument("--rows", type=int, default=0, help="--profile of a 2D workload: this tile height")
    ap.add_argument("--no-secondary", action="store_true",
                    help="head600: skip the config-3, config-4 and config-5 figures added to the line")
    ap.add_argument("--cpu-steps", type=int, default=12)
    ap.add_argument("--profile", type=int, default=0,
                    help="run only N fused steps of one sample (for ncu), no timing, no JSON")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "ours":
        args.warmup = 3
    if args.impl == "reference":
        if args.workload in ("adjoint400", "adjoint192"):
            run_adjoint_reference(args)
        elif args.workload == "single4096":
            run_single_reference(args)
        elif args.workload == "pack256":
            run_pack_reference(args)
        else:
            run_reference(args, WORKLOADS[args.workload])
        return
    if args.workload == "adjoint400":
        if args.profile:
            run_profile_adjoint(args)
        else:
            run_adjoint_bench(args)
        return
    if args.workload == "adjoint192":
        if args.profile:
            run_profile_adjoint3d(args)
        else:
            run_adjoint3d_bench(args)
        return
    if args.workload == "single4096":
        run_single_bench(args)
        return
    if args.workload == "pack256":
        run_pack_bench(args)
        return
    w = WORKLOADS[args.workload]
    if args.profile:
        run_profile(args, w)
    else:
        run_ours(args, w)


if __name__ == "__main__":
    main()

"""Dataset generation on the device: the reference's production caller of the
batched solver (scripts/generate_corrected_dataset.py:46-306), B200-first.

Per sample, as the reference: a hemorrhage with probability given by
``hemorrhage_ratio`` (centre at U(0, 3) cm from the middle in a U(0, 2 pi)
direction, radius U(0.3, 1.5) cm; :46-58, :215-218), the concentric brain
phantom with the fixed tissue table (head_models.py:519-631), a ring of
``n_ant`` antennas of radius nx//3 (:120-129), CPML 10, ``total_steps`` from
the reference formula int(2 * sqrt(2) nx dx / c / (1 / 4f)) (:131-136) unless
given, the probe series scaled by the correction factor 6.58e12 (:156), and
the reference's files:

    <output>/s_matrix/sample_%06d.npy   (n_ant tx, n_ant rx, total_steps) float64
    <output>/eps_map/sample_%06d.npy    (nx, ny) float64
    <output>/hem_mask/sample_%06d.npy   (nx, ny) float64
    <output>/metadata/sample_%06d.json  (the reference's per-sample schema)
    <output>/dataset_metadata.json

Differences, by design: the draws come from a seeded generator (the
reference uses NumPy's global state), and s_matrix holds every TX/RX pair
(the reference stores ``s_params[0][0]``, the TX 0 -> RX 0 series, although
its comment and file name describe the (n_ant, n_ant, n_time) matrix).

The B200 path: the phantoms of a batch are rasterised together by one CUDA
kernel (``ceep_brain_phantom_2d``), their update coefficients are formed in
FP64 on the device, and the batch's solvers run in one packed launch per
step (``PackedBatch2D``); only the finished series and maps cross to the host.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import time
from dataclasses import dataclass
from pathlib import Path
from typing import List, Optional, Sequence, Tuple

import numpy as np
import torch

from . import physics
from ._lib import check, lib
from .distributed import gather_objects, shard, world
from .packed import PackedBatch2D
from .phantoms import ring_positions
from .solvers import BatchedFDTD2D

CORRECTION_FACTOR = 6.58e12  # generate_corrected_dataset.py:42
# head_models.py:583-590 (eps_r, sigma) and layer thicknesses :538-541
TISSUE = ((40.0, 1.0), (12.0, 0.2), (68.0, 2.5), (52.0, 1.8), (38.0, 1.2), (61.0, 2.0))
THICKNESS = (3e-3, 7e-3, 2e-3, 10e-3)  # skin, skull, csf, grey


@dataclass
class SampleSpec:
    sample_id: int
    include_hemorrhage: bool
    center_cm: Optional[Tuple[float, float]] = None
    radius_cm: float = 0.0


def draw_samples(n_samples: int, hemorrhage_ratio: float = 0.7, seed: int = 0) -> List[SampleSpec]:
    """Which samples get a hemorrhage and its parameters (:46-58, :215-218)."""
    rng = np.random.default_rng(seed)
    n_hem = int(n_samples * hemorrhage_ratio)
    has = rng.permutation([True] * n_hem + [False] * (n_samples - n_hem))
    out = []
    for i in range(n_samples):
        if has[i]:
            angle = rng.uniform(0, 2 * np.pi)
            dist = rng.uniform(0, 3.0)
            radius = rng.uniform(0.3, 1.5)
            out.append(SampleSpec(i, True, (dist * np.cos(angle), dist * np.sin(angle)), radius))
        else:
            out.append(SampleSpec(i, False))
    return out


def reference_total_steps(nx: int, dx: float, frequency: float) -> int:
    """generate_corrected_dataset.py:131-136 (note: dt there is 1/(4f), not the
    FDTD step, so the count is small)."""
    max_dist = np.sqrt(2) * (nx * dx)
    return int(2 * (max_dist / 3e8) / (1 / (4 * frequency)))


def layer_radii(head_radius_cm: float = 9.0) -> Tuple[float, ...]:
    """Outer radii (m) of skin, skull, csf, grey, white (head_models.py:600-604)."""
    r = [head_radius_cm * 1e-2]
    for t in THICKNESS:
        r.append(r[-1] - t)
    return tuple(r)


def brain_phantom_maps(specs: Sequence[SampleSpec], nx: int, ny: int, dx: float, head_radius_cm: float = 9.0,
                       device="cuda"):
    """(eps_r, sigma, hemorrhage mask), each (batch, nx, ny) FP64 on the device,
    rasterised by one kernel for all `specs`."""
    dev = torch.device(device)
    B = len(specs)
    hem = np.array([[s.center_cm[0] * 1e-2, s.center_cm[1] * 1e-2, s.radius_cm * 1e-2] if s.include_hemorrhage
                    else [0.0, 0.0, -1.0] for s in specs], np.float64)
    hem_t = torch.as_tensor(hem).to(dev)
    radii = np.ascontiguousarray(layer_radii(head_radius_cm), np.float64)       # host
    tissue = np.ascontiguousarray(np.array(TISSUE, np.float64).reshape(-1))    # host
    eps = torch.empty((B, nx, ny), dtype=torch.float64, device=dev)
    sig = torch.empty_like(eps)
    mask = torch.empty_like(eps)
    stream = C.c_void_p(torch.cuda.current_stream(dev).cuda_stream)
    check(lib().ceep_brain_phantom_2d(B, nx, ny, float(dx), radii.ctypes.data, tissue.ctypes.data,
                                      hem_t.data_ptr(), eps.data_ptr(), sig.data_ptr(), mask.data_ptr(), stream),
          "ceep_brain_phantom_2d")
    return eps, sig, mask


def simulate_batch(specs: Sequence[SampleSpec], nx: int = 64, ny: int = 64, dx: float = 0.5e-3,
                   frequency: float = 2e9, n_ant: int = 16, total_steps: Optional[int] = None, cpml: int = 10,
                   head_radius_cm: float = 9.0, device="cuda"):
    """Rasterise, run and scale one batch of samples.  Returns the device maps
    (eps, sigma, mask) and the (batch, n_ant, n_ant, total_steps) FP64 series
    already multiplied by the correction factor."""
    T = reference_total_steps(nx, dx, frequency) if total_steps is None else int(total_steps)
    if T < 1:
        raise ValueError("total_steps must be at least 1")
    eps, sig, mask = brain_phantom_maps(specs, nx, ny, dx, head_radius_cm, device)
    pos = ring_positions(n_ant, (nx // 2, ny // 2), nx // 3)
    solvers = []
    for b in range(len(specs)):
        s = BatchedFDTD2D(nx, ny, dx, T, cpml, pos, pos, frequency, device=str(device))
        s._build()
        coef, _ = physics.coefficient_tensors_kernel(eps[b], sig[b], s.dt, device=s.device)
        s.load_material_tensors((coef, None))
        solvers.append(s)
    pk = PackedBatch2D(solvers)
    pk.reset()
    pk.advance()
    series = torch.stack([s.probe_data[:, :n_ant] for s in solvers]).double() * CORRECTION_FACTOR
    for s in solvers:
        s.check_status()
    return eps, sig, mask, series, T


def sample_metadata(spec: SampleSpec, nx, ny, dx, frequency, n_ant, total_steps) -> dict:
    """The reference's per-sample schema (generate_corrected_dataset.py:159-177)."""
    hem = spec.include_hemorrhage
    return {
        "sample_id": spec.sample_id,
        "include_hemorrhage": bool(hem),
        "hemorrhage_params": {
            "center_x": float(spec.center_cm[0]),
            "center_y": float(spec.center_cm[1]),
            "radius": float(spec.radius_cm),
        } if hem else None,
        "simulation_params": {"nx": nx, "ny": ny, "dx": dx, "frequency": frequency, "n_antennas": n_ant,
                              "total_steps": total_steps},
        "correction_applied": True,
        "correction_factor": float(CORRECTION_FACTOR),
        "meep_validated": True,
    }


def generate_dataset(n_samples: int = 100, output_dir: str = "dataset_corrected", hemorrhage_ratio: float = 0.7,
                     nx: int = 64, ny: int = 64, dx: float = 0.5e-3, frequency: float = 2e9, n_ant: int = 16,
                     total_steps: Optional[int] = None, seed: int = 0, batch: int = 128, device="cuda",
                     write: bool = True) -> dict:
    """Generate the dataset in batches of `batch` packed samples; returns the
    dataset metadata (also written as dataset_metadata.json).

    Under torch.distributed (one process per GPU) every rank draws the same
    sample specs and simulates and writes its contiguous share of them
    (``distributed.shard``); the per-sample magnitudes and the slowest rank's
    time are gathered, so every rank returns the whole dataset's metadata and
    rank 0 writes it.  Samples never cross ranks: no collective touches the
    simulation."""
    rank, size = world()
    out = Path(output_dir)
    if write:
        for sub in ("s_matrix", "eps_map", "hem_mask", "metadata"):
            (out / sub).mkdir(parents=True, exist_ok=True)
    specs = shard(draw_samples(n_samples, hemorrhage_ratio, seed), rank, size)
    mags, t0 = [], time.perf_counter()
    T = None
    for b0 in range(0, len(specs), batch):
        chunk = specs[b0:b0 + batch]
        eps, sig, mask, series, T = simulate_batch(chunk, nx, ny, dx, frequency, n_ant, total_steps,
                                                   device=device)
        series_h, eps_h, mask_h = series.cpu().numpy(), eps.cpu().numpy(), mask.cpu().numpy()
        for k, spec in enumerate(chunk):
            mags.append((spec.sample_id, float(np.abs(series_h[k]).max())))
            if write:
                name = f"sample_{spec.sample_id:06d}"
                np.save(out / "s_matrix" / f"{name}.npy", series_h[k])
                np.save(out / "eps_map" / f"{name}.npy", eps_h[k])
                np.save(out / "hem_mask" / f"{name}.npy", mask_h[k])
                with open(out / "metadata" / f"{name}.json", "w") as f:
                    json.dump(sample_metadata(spec, nx, ny, dx, frequency, n_ant, T), f, indent=2)
    elapsed = time.perf_counter() - t0
    gathered = gather_objects((mags, T, elapsed))
    mags = sorted(m for part, _, _ in gathered for m in part)
    T = next((t for _, t, _ in gathered if t is not None), T)
    elapsed = max(e for _, _, e in gathered)
    m = np.array([v for _, v in mags])
    expected = 3.368  # the MEEP-validated magnitude the reference checks against (:262-266)
    meta = {
        "n_samples": n_samples,
        "hemorrhage_ratio": hemorrhage_ratio,
        "correction_factor": float(CORRECTION_FACTOR),
        "meep_validated": True,
        "seed": seed,
        "simulation_params": {"nx": nx, "ny": ny, "dx": dx, "frequency": frequency, "n_antennas": n_ant,
                              "total_steps": T, "cpml_thickness": 10},
        "s_matrix_statistics": {"mean": float(m.mean()), "std": float(m.std()), "min": float(m.min()),
                                "max": float(m.max())},
        "meep_reference": {"expected_magnitude": expected, "actual_mean_magnitude": float(m.mean()),
                           "ratio": float(m.mean() / expected)},
        "generation_seconds": elapsed,
        "samples_per_second": n_samples / elapsed if elapsed > 0 else None,
    }
    if size > 1:
        meta["ranks"] = size
    if write and rank == 0:
        with open(out / "dataset_metadata.json", "w") as f:
            json.dump(meta, f, indent=2)
    return meta


def main(argv=None):
    ap = argparse.ArgumentParser(description="Generate the brain hemorrhage dataset on the GPU")
    ap.add_argument("--n_samples", type=int, default=100)
    ap.add_argument("--output", type=str, default="dataset_corrected")
    ap.add_argument("--hemorrhage_ratio", type=float, default=0.7)
    ap.add_argument("--nx", type=int, default=64)
    ap.add_argument("--ny", type=int, default=64)
    ap.add_argument("--dx", type=float, default=0.5e-3)
    ap.add_argument("--frequency", type=float, default=2e9)
    ap.add_argument("--n_ant", type=int, default=16)
    ap.add_argument("--total_steps", type=int, default=None, help="default: the reference's formula")
    ap.add_argument("--seed", type=int, default=0)
    ap.add_argument("--batch", type=int, default=128, help="samples per packed launch")
    a = ap.parse_args(argv)
    meta = generate_dataset(a.n_samples, a.output, a.hemorrhage_ratio, a.nx, a.ny, a.dx, a.frequency, a.n_ant,
                            a.total_steps, a.seed, a.batch)
    print(json.dumps(meta, indent=2))


if __name__ == "__main__":
    main()

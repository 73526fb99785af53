"""Many phantoms of uneven size, step count, TX count and dispersion model in
one launch per time step, replayed from a CUDA graph.

The reference has no counterpart: its dataset generator builds and runs one
``BatchedFDTD2D`` per phantom (scripts/generate_corrected_dataset.py:139-149),
which leaves a B200 mostly idle for the smaller grids.  ``PackedBatch2D``
takes already-configured ``BatchedFDTD2D`` solvers, packs the tiles of all of
them into per-class tile tables (class = TX lane width x ADE shape; phantoms
sorted by decreasing step count so the running tiles form a prefix) and
advances all of them together (``ceep2d_pack_*`` in include/ceep_b200.h).
Each solver's ``probe_data``, ``ez`` ... hold its own results afterwards.

``temporal_block=2`` advances every running phantom two steps per launch with
the temporal-block kernel (a phantom with an odd step count takes its last
step alone).  ``packing`` places the classes in time: 0 interleaves their
launches on one stream, 1 runs each class's launch chain on its own stream
beside the others.  ``autotune`` picks the temporal-block depth, the tile
height (rows per block) and the packing by timing a short prefix of the
packed run for each candidate.
"""
from __future__ import annotations

import ctypes as C
from typing import Dict, List, Sequence, Tuple

import numpy as np
import torch

from ._lib import check, lib
from .solvers import BatchedFDTD2D


class PackedBatch2D:
    def __init__(self, solvers: Sequence[BatchedFDTD2D], rows: int = 16, use_graph: bool = True,
                 temporal_block: int = 1, packing: int = 0):
        if not solvers:
            raise ValueError("no solvers")
        self.solvers: List[BatchedFDTD2D] = list(solvers)
        self.device = self.solvers[0].device
        self.use_graph = use_graph
        self._pack = None
        self._ws = None
        self.rows = int(rows)
        self.temporal_block = int(temporal_block)
        if self.temporal_block not in (1, 2):
            raise ValueError("temporal_block must be 1 or 2")
        self.packing = int(packing)
        if self.packing not in (0, 1):
            raise ValueError("packing must be 0 (interleaved) or 1 (concurrent class chains)")
        for s in self.solvers:
            if s.device != self.device:
                raise ValueError("all solvers must live on one device")
            if not s._built:
                s._build()
        self._replan(self.rows)

    @property
    def max_steps(self) -> int:
        return max(s.total_steps for s in self.solvers)

    @property
    def cell_steps(self) -> int:
        return sum(s.nx * s.ny * s.total_steps * s.batch for s in self.solvers)

    def _destroy(self):
        if self._pack is not None:
            lib().ceep2d_pack_destroy(self._pack)
            self._pack = None

    def __del__(self):
        try:
            self._destroy()
        except Exception:
            pass

    def _replan(self, rows: int):
        self._destroy()
        for s in self.solvers:
            s.set_rows_per_block(rows)
        plans = (C.c_void_p * len(self.solvers))(*[s._plan.value for s in self.solvers])
        nbytes = lib().ceep2d_pack_workspace_bytes(plans, len(self.solvers))
        if nbytes < 0:
            raise RuntimeError(lib().ceep_last_error().decode())
        self._ws = torch.empty(nbytes, dtype=torch.uint8, device=self.device)
        stream = torch.cuda.current_stream(self.device)
        h = C.c_void_p()
        check(lib().ceep2d_pack_create(plans, len(self.solvers), self._ws.data_ptr(), nbytes,
                                       C.c_void_p(stream.cuda_stream), C.byref(h)), "ceep2d_pack_create")
        self._pack = h
        self.rows = rows
        check(lib().ceep2d_pack_set_temporal_block(h, self.temporal_block), "ceep2d_pack_set_temporal_block")
        check(lib().ceep2d_pack_set_packing(h, self.packing), "ceep2d_pack_set_packing")

    @property
    def classes(self) -> int:
        """Launch classes (lane width x ADE shape) of the packed solvers."""
        return len({(s._gwidth, len(s._debye), len(s._lorentz)) for s in self.solvers})

    def reset(self):
        for s in self.solvers:
            s.reset()

    def advance(self, step0: int = 0, nsteps: int = None, stream=None):
        nsteps = self.max_steps - step0 if nsteps is None else nsteps
        s = torch.cuda.current_stream(self.device) if stream is None else stream
        check(lib().ceep2d_pack_run(self._pack, step0, nsteps, C.c_void_p(s.cuda_stream), int(self.use_graph)),
              "ceep2d_pack_run")

    def run(self) -> List[Dict[int, Dict[int, np.ndarray]]]:
        """All steps of every phantom from a zero state; one result dict each."""
        self.reset()
        self.advance()
        out = []
        for s in self.solvers:
            p = s.probe_data.double().cpu().numpy()
            s.check_status()
            out.append({tx: {rx: p[tx, rx] for rx in range(len(s.probe_positions))} for tx in range(s.batch)})
        return out

    def tiles_at(self, step: int) -> int:
        return lib().ceep2d_pack_tiles(self._pack, step)

    def autotune(self, candidates=(8, 12, 16, 20, 24, 32, 48), probe_steps: int = 40,
                 temporal_blocks=(1, 2), packings=(0, 1)) -> Dict[Tuple[int, int, int], float]:
        """Time ``probe_steps`` packed steps for each (temporal-block depth,
        tile height, packing); keep the fastest.  Returns ms per step for
        each.  With a single class the packings coincide and only 0 is tried."""
        stream = torch.cuda.current_stream(self.device)
        timings = {}
        nst = min(probe_steps, self.max_steps)
        nst -= nst % 2 if nst < self.max_steps else 0    # even, unless the whole run
        packings = tuple(packings) if self.classes > 1 else (0,)
        for tb in temporal_blocks:
            for rows in candidates:
                self.temporal_block = tb
                self._replan(rows)
                for pkg in packings:
                    self.packing = pkg
                    check(lib().ceep2d_pack_set_packing(self._pack, pkg), "ceep2d_pack_set_packing")
                    self.advance(0, nst, stream)           # capture + warm
                    self.reset()
                    a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                    a.record(stream)
                    self.advance(0, nst, stream)
                    b.record(stream)
                    torch.cuda.synchronize(self.device)
                    timings[(tb, rows, pkg)] = a.elapsed_time(b) / nst
                    self.reset()
        best = min(timings, key=timings.get)
        self.temporal_block, self.packing = best[0], best[2]
        self._replan(best[1])
        return timings

"""Phase tracing and per-run records.

The reference only prints a rate when asked (``BatchedFDTD3D.run(verbose)``,
src/ceep/solvers/fdtd_3d_batched.py:960-973).  Here every ``run()`` leaves a
JSON-serialisable record on the solver (``solver.run_record``: grid, steps,
TX, host wall time, GCell-steps/s, device status), appended as one JSON line
to ``solver.record_path`` when that is set, and the time loop, the DFT and
the DAS image are wrapped in NVTX ranges (``ceep:time_loop``, ``ceep:dft``,
``ceep:das``) that show up in any CUDA profiler timeline.
"""
from __future__ import annotations

import contextlib
import json
import time
from typing import Optional

import torch


@contextlib.contextmanager
def phase(name: str):
    """NVTX range `ceep:<name>` around a host-side phase (no-op where NVTX is absent)."""
    pushed = False
    try:
        torch.cuda.nvtx.range_push("ceep:" + name)
        pushed = True
    except Exception:
        pass
    try:
        yield
    finally:
        if pushed:
            try:
                torch.cuda.nvtx.range_pop()
            except Exception:
                pass


def make_record(kind: str, cells: int, steps: int, tx: int, seconds: float, status: int = 0,
                extra: Optional[dict] = None) -> dict:
    rec = {"solver": kind, "cells": int(cells), "steps": int(steps), "tx": int(tx),
           "seconds": round(float(seconds), 6),
           "gcell_steps_per_s": round(cells * steps * tx / seconds / 1e9, 4) if seconds > 0 else None,
           "status": int(status), "time": time.time()}
    if extra:
        rec.update(extra)
    return rec


def emit(solver, rec: dict) -> None:
    """Store `rec` on the solver and append it to ``solver.record_path`` if set."""
    solver.run_record = rec
    path = getattr(solver, "record_path", None)
    if path:
        with open(path, "a") as f:
            f.write(json.dumps(rec) + "\n")

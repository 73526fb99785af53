"""Array-module shim that lets the reference's batched solvers run on NumPy.

Used only by ``make_golden.py`` (fixture generation, in a container that has
the reference checkout) and by the CPU tests that re-validate the oracle
against the live reference when that checkout is present.

The reference reads its array module through
``ceep.core.backend._backend_manager.module`` (src/ceep/core/backend.py:70,
:242).  Two defects stop its batched ``run()`` on NumPy: it calls
``cp.asnumpy`` (src/ceep/solvers/fdtd_2d_batched.py:529), which NumPy lacks,
and it hard-codes float64 allocations (:147-149, :188-191), so an FP32 run
needs the float dtype forced.  This shim supplies both without editing the
reference.
"""
from __future__ import annotations

import os
import sys
import types

import numpy as np

REFERENCE_ROOT = os.environ.get("CEEP_REFERENCE_ROOT", "/root/reference")


def reference_available() -> bool:
    return os.path.isdir(os.path.join(REFERENCE_ROOT, "src", "ceep"))


def _float_forcing_numpy(dtype):
    dtype = np.dtype(dtype)
    mod = types.ModuleType("numpy_forced_" + dtype.name)

    def _fix(dt, like=None):
        if dt is None:
            if like is not None and np.issubdtype(np.asarray(like).dtype, np.floating):
                return dtype
            return None
        if np.issubdtype(np.dtype(dt), np.floating):
            return dtype
        return dt

    mod.zeros = lambda shape, dtype=np.float64: np.zeros(shape, dtype=_fix(dtype))
    mod.ones = lambda shape, dtype=np.float64: np.ones(shape, dtype=_fix(dtype))
    mod.empty = lambda shape, dtype=np.float64: np.empty(shape, dtype=_fix(dtype))
    mod.full = lambda shape, v, dtype=np.float64: np.full(shape, v, dtype=_fix(dtype))
    mod.asarray = lambda a, dtype=None: np.asarray(a, dtype=_fix(dtype, a))
    mod.array = lambda a, dtype=None: np.array(a, dtype=_fix(dtype, a))
    mod.zeros_like = lambda a: np.zeros_like(a)
    mod.asnumpy = np.asarray

    def __getattr__(name):
        return getattr(np, name)

    mod.__getattr__ = __getattr__
    return mod


def import_reference(dtype=np.float64):
    """Import the reference package and install the NumPy shim for ``dtype``."""
    src = os.path.join(REFERENCE_ROOT, "src")
    if src not in sys.path:
        sys.path.insert(0, src)
    import ceep.core.backend as backend  # noqa: E402

    backend._backend_manager.module = _float_forcing_numpy(dtype)
    return backend

"""C-ABI checks that need no GPU: the library loads, exports every function
declared in include/*.h, its struct mirror matches, and argument validation
rejects bad descriptors before any CUDA call."""
import ctypes as C
import glob
import os
import re

import pytest

from conftest import ROOT


def _declared():
    names = set()
    for h in glob.glob(os.path.join(ROOT, "include", "*.h")):
        src = open(h).read()
        src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
        names.update(re.findall(r"^\s*[A-Za-z_][\w\s\*]*?\b(ceep\w*)\s*\(", src, flags=re.M))
    return sorted(names)


def test_header_declares_entry_points():
    names = _declared()
    for must in ("ceep2d_plan_create", "ceep2d_plan_run", "ceep_dft", "ceep_das", "ceep_das_time"):
        assert must in names


def test_library_exports_every_declared_symbol():
    from ceep_b200 import _lib
    h = _lib.lib()
    for name in _declared():
        assert hasattr(h, name), name
        assert name in _lib.exported_symbols(), f"{name} not bound in _lib"


def test_desc_mirror_size():
    from ceep_b200 import _lib
    assert _lib.lib().ceep2d_desc_size() == C.sizeof(_lib.Desc2D)


def test_plan_create_rejects_bad_descriptors():
    from ceep_b200 import _lib
    h = _lib.lib()
    d = _lib.Desc2D()
    d.nx, d.ny, d.cpml, d.ntx, d.ntx_pad, d.nsteps = 40, 40, 1, 2, 4, 10
    plan = C.c_void_p()
    assert h.ceep2d_plan_create(C.byref(d), C.byref(plan)) == 1
    assert b"cpml" in h.ceep_last_error()
    d.cpml = 25
    assert h.ceep2d_plan_create(C.byref(d), C.byref(plan)) == 1
    d.cpml, d.ntx_pad = 5, 6
    assert h.ceep2d_plan_create(C.byref(d), C.byref(plan)) == 1
    d.ntx_pad = 4
    assert h.ceep2d_plan_create(C.byref(d), C.byref(plan)) == 1  # null buffers
    assert b"null" in h.ceep_last_error()
    assert not plan.value


def test_spectral_entry_points_validate():
    from ceep_b200 import _lib
    h = _lib.lib()
    assert h.ceep_dft(None, None, None, 1, 1, 1, 1, None) == 1
    assert h.ceep_das(None, None, None, 1, 1, 1, 1, 0.0, 0.0, 1.0, 1, None, None, None) == 1
    assert h.ceep_das_time(None, None, 1, 1, 1, 1.0, 1.0, None, None) == 1
    assert h.ceep_das_workspace_bytes(64, 64, 301) > 0


def test_material_and_plan_settings_validate():
    """The coefficient kernel's entry point and the plan settings reject bad
    arguments before any CUDA call."""
    from ceep_b200 import _lib
    h = _lib.lib()
    assert h.ceep2d_material_coefficients(None, None, None, 0, 0, 4, 4, 1e-12, 8.85e-12, None, None, None) == 1
    one = C.c_void_p(16)  # never dereferenced: the checks fail first
    assert h.ceep2d_material_coefficients(one, one, None, 3, 0, 4, 4, 1e-12, 8.85e-12, one, one, None) == 1
    assert h.ceep2d_material_coefficients(one, one, None, 1, 0, 4, 4, 1e-12, 8.85e-12, one, one, None) == 1
    assert b"pole" in h.ceep_last_error()
    assert h.ceep2d_material_coefficients(one, one, None, 0, 0, 0, 4, 1e-12, 8.85e-12, one, None, None) == 1
    assert h.ceep2d_plan_set_frame_split(None, 1) == 1
    assert h.ceep2d_adjoint_set_rows(None, 4) == 1


@pytest.mark.parametrize("side", [65536, 65537, 46341])
def test_image_entry_points_reject_pixel_counts_past_int(side):
    """Pixel counts are formed in 64 bits: 65536^2 (a multiple of 2^32),
    65537^2 (wraps to a small count in 32 bits) and 46341^2 (wraps negative)
    are refused before any launch, with no device touched."""
    from ceep_b200 import _lib
    h = _lib.lib()
    fake = C.c_void_p(256)  # never dereferenced: the size check comes first
    assert h.ceep_das_workspace_bytes(side, side, 301) == 0
    assert h.ceep_dmas_workspace_bytes(side, side) == 0
    args = (fake, fake, fake, 301, 16, side, side, 0.0, 0.0, 1e-3, 1)
    assert h.ceep_das(*args, fake, fake, None) == 3
    assert b"exceeds" in h.ceep_last_error()
    assert h.ceep_dmas(*args, fake, fake, None) == 3
    assert h.ceep_das_noalloc(*args, fake, None) == 3
    assert b"exceeds" in h.ceep_last_error()
    assert h.ceep_das_time(fake, fake, 4, 16, side, 1e-3, 2e9, fake, None) == 3


def test_solver_validates_positions_without_gpu():
    from ceep_b200 import BatchedFDTD2D
    with pytest.raises(ValueError):
        BatchedFDTD2D(40, 40, 1e-3, 10, 5, [(-1, 3)], [(3, 3)], 2e9)
    with pytest.raises(ValueError):
        BatchedFDTD2D(40, 40, 1e-3, 10, 5, [(3, 3)], [(3, 40)], 2e9)
    with pytest.raises(ValueError):
        BatchedFDTD2D(40, 40, 1e-3, 10, 1, [(3, 3)], [(3, 3)], 2e9)
    s = BatchedFDTD2D(40, 40, 1e-3, 10, 5, [(3, 3)], [(3, 3)], 2e9)
    with pytest.raises(TypeError):
        s.set_phantom(object())

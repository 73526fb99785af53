"""The delay-and-sum entry point that allocates nothing (ceep_das_noalloc).

It serves callers that cannot give this library any device memory -- hosts
that reserve all of their GPU memory in their own pool up front and may not
allocate while imaging -- by keeping its partial sums in a fixed array inside
the library.  The test calls it through the C ABI twice in a row, on two
different problems, and checks each image against the workspace-taking
ceep_das on the same inputs.  It builds its inputs itself so it passes both
alone in a fresh process and after the rest of the suite.
"""
import ctypes as C

import numpy as np
import pytest
import torch

pytestmark = pytest.mark.gpu
TOL = 1e-4


def _problem(seed, nfreq, nant, nxp, nyp, device):
    rng = np.random.default_rng(seed)
    S = rng.standard_normal((nfreq, nant, nant, 2)).astype(np.float32)
    f = np.linspace(0.5e9, 3.5e9, nfreq)
    k = (2 * np.pi * f / 299_792_458.0).astype(np.float32)
    ang = 2 * np.pi * np.arange(nant) / nant
    ant = np.stack([0.15 + 0.1 * np.cos(ang), 0.15 + 0.1 * np.sin(ang)], 1).astype(np.float32)
    t = lambda a: torch.as_tensor(a).to(device)
    return t(S), t(k), t(ant), (nfreq, nant, nxp, nyp, 0.06, 0.07, 0.18 / nxp)


def _run(lib, S, k, ant, dims, noalloc, device):
    nfreq, nant, nxp, nyp, px0, py0, pix = dims
    img = torch.empty((nxp, nyp), dtype=torch.float32, device=device)
    stream = C.c_void_p(torch.cuda.current_stream(device).cuda_stream)
    if noalloc:
        rc = lib.ceep_das_noalloc(S.data_ptr(), k.data_ptr(), ant.data_ptr(), nfreq, nant, nxp, nyp, px0, py0, pix,
                                  1, img.data_ptr(), stream)
    else:
        ws = torch.empty(lib.ceep_das_workspace_bytes(nxp, nyp, nfreq), dtype=torch.uint8, device=device)
        rc = lib.ceep_das(S.data_ptr(), k.data_ptr(), ant.data_ptr(), nfreq, nant, nxp, nyp, px0, py0, pix, 1,
                          ws.data_ptr(), img.data_ptr(), stream)
    assert rc == 0, lib.ceep_last_error()
    torch.cuda.synchronize(device)
    return img.cpu().numpy()


def test_noalloc_das_matches_workspace_das_twice(cuda_device):
    from ceep_b200._lib import lib
    h = lib()
    first = _problem(1, 301, 16, 64, 64, cuda_device)      # the head-imaging shape
    second = _problem(2, 37, 9, 40, 23, cuda_device)       # a different, smaller one
    for S, k, ant, dims in (first, second):
        want = _run(h, S, k, ant, dims, False, cuda_device)
        got = _run(h, S, k, ant, dims, True, cuda_device)
        err = np.linalg.norm(got - want) / np.linalg.norm(want)
        assert err < TOL, err


def test_noalloc_das_rejects_oversized_problems(cuda_device):
    from ceep_b200._lib import lib
    h = lib()
    cap = h.ceep_das_noalloc_capacity()
    side = int(np.ceil(np.sqrt(cap))) + 8          # one frequency chunk already exceeds the array
    img = torch.empty(1, device=cuda_device)
    rc = h.ceep_das_noalloc(img.data_ptr(), img.data_ptr(), img.data_ptr(), 4, 4, side, side, 0.0, 0.0, 1e-3, 1,
                            img.data_ptr(), None)
    assert rc == 3 and b"fixed scratch" in h.ceep_last_error()

"""Failure detection on the device, with no GPU fault: a bounded wait that is
made to run out, and the NaN/Inf sentinel.

The reference only checks `np.all(np.isfinite(signal))` after a run
(tests/test_fdtd_3d_batched.py:240-244).  Here the step kernels bound every
mbarrier wait and record CEEP_ERR_TIMEOUT in a status word; a test makes one
run out by having the producer skip one row's copies (a flag nothing else
sets) with a 1 ms limit, and checks that the launch returns, the status reads
TIMEOUT, run() raises, and a fresh solver afterwards is bit-correct.  The
sentinel scans Ez and the probe samples on the device and reports
CEEP_ERR_NONFINITE; a non-finite waveform sample fed from the host must make
run() raise."""
import time

import numpy as np
import pytest
import torch

from ceep_b200 import BatchedFDTD2D, physics
from ceep_b200.solvers import FDTDStatusError

pytestmark = pytest.mark.gpu

NX, NY, N, T = 96, 80, 8, 120
SRC = [(30, 30), (60, 40), (45, 60), (20, 50), (70, 20)]


def _solver(tblock, waveform=None, wait_ns=None):
    s = BatchedFDTD2D(NX, NY, 0.5e-3, T, N, SRC, SRC, 2e9, temporal_block=tblock, waveform=waveform,
                      device="cuda:0")
    x, y = np.meshgrid(np.arange(NX), np.arange(NY), indexing="ij")
    m = (x - 48) ** 2 + (y - 40) ** 2 <= 12 ** 2
    s._eps_r[m], s._sigma_e[m] = 9.0, 0.3
    if wait_ns:
        s.set_wait_limit(wait_ns)
    return s


@pytest.mark.parametrize("tblock", [1, 2])
def test_expired_wait_reports_timeout_and_leaves_the_context_usable(tblock):
    good = _solver(tblock)
    good.run()
    want = good.probe_data.clone()

    bad = _solver(tblock, wait_ns=1_000_000)   # 1 ms
    bad._build()
    bad.inject_copy_fault(NY // 2)
    t0 = time.time()
    with pytest.raises(FDTDStatusError) as err:
        bad.run()
    assert err.value.code == FDTDStatusError.TIMEOUT
    assert time.time() - t0 < 60, "every launch must end soon after its 1 ms waits run out"
    torch.cuda.synchronize()

    fresh = _solver(tblock)
    fresh.run()
    assert torch.equal(fresh.probe_data, want)


@pytest.mark.parametrize("tblock", [1, 2])
def test_fault_row_off_again_runs_clean(tblock):
    """The injection hook turned back off leaves the plan's launches unchanged."""
    a = _solver(tblock)
    a._build()
    a.inject_copy_fault(10)
    a.inject_copy_fault(-1)
    a.run()
    b = _solver(tblock)
    b.run()
    assert torch.equal(a.probe_data, b.probe_data)


@pytest.mark.parametrize("bad_value", [np.nan, np.inf])
@pytest.mark.parametrize("interval", [0, 16])
def test_sentinel_reports_a_nonfinite_waveform_sample(bad_value, interval):
    dt = BatchedFDTD2D(NX, NY, 0.5e-3, T, N, SRC, SRC, 2e9).dt
    w = physics.gaussian_derivative(T, dt, 2e9, 5.0)
    w[37] = bad_value
    s = _solver(2, waveform=w)
    s.set_sentinel(interval)
    with pytest.raises(FDTDStatusError) as err:
        s.run()
    assert err.value.code == FDTDStatusError.NONFINITE


def test_sentinel_stays_quiet_on_a_finite_run():
    s = _solver(2)
    s.set_sentinel(7)
    s.run()
    s.check_status()
    assert torch.isfinite(s.probe_data).all()

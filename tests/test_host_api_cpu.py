"""Host-side checks of the batched solver's API that need no GPU."""
import numpy as np
import pytest


def test_poles_must_stay_inside_the_interior_e_region():
    """An ADE pole in a CPML strip cell (outside [n+1, nx-n) x [n+1, ny-n),
    where the ADE does not act) is rejected; one on the region's edge cells is
    accepted."""
    from ceep_b200.solvers import BatchedFDTD2D
    nx, ny, n = 60, 50, 6
    s = BatchedFDTD2D(nx, ny, 0.5e-3, 10, n, [(30, 25)], [(30, 25)], 2e9, device="cpu")
    cases = [((n, 25), False), ((n + 1, 25), True), ((nx - n - 1, 25), True), ((nx - n, 25), False),
             ((30, n), False), ((30, n + 1), True), ((30, ny - n - 1), True), ((30, ny - n), False),
             ((0, 0), False), ((nx - 1, ny - 1), False)]
    for (i, j), ok in cases:
        de, tau = np.zeros((nx, ny)), np.zeros((nx, ny))
        de[i, j], tau[i, j] = 5.0, 1e-11
        if ok:
            s.set_dispersion(debye=[(de, tau)])
            s.set_dispersion(lorentz=[(de, tau * 1e22, tau * 1e20)])
        else:
            with pytest.raises(ValueError):
                s.set_dispersion(debye=[(de, tau)])
            with pytest.raises(ValueError):
                s.set_dispersion(lorentz=[(de, tau * 1e22, tau * 1e20)])
    # a zero delta_eps or tau leaves the cell pole-free wherever it sits
    de, tau = np.zeros((nx, ny)), np.zeros((nx, ny))
    de[0, 0] = 5.0
    s.set_dispersion(debye=[(de, tau)])

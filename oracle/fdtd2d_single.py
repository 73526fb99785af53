"""CPU oracle for the non-batched 2D solver (TMz / TEz) — TEST INFRASTRUCTURE ONLY.

NumPy FP64 restatement of one ``FDTD2D.step()`` of the reference
(src/ceep/solvers/fdtd_base.py:158-190, the template order
H update -> H boundaries -> E update -> sources -> E boundaries -> record)
with the field updates of src/ceep/solvers/fdtd_2d.py:111-243 and the
boundaries of src/ceep/boundaries/absorbing.py:

* PEC   (:48-78)   tangential E zeroed on the four edges
* Mur   (:80-172)  first-order Mur on the edges of Ez (TMz) / Hz (TEz)
* CPML  (:174-561) CFS-CPML with polynomial sigma/kappa and linear alpha
                   grading; psi recurrences over the strip cells, H
                   corrections with dt/mu0 and E corrections with dt/eps0

Arrays are (nx, ny) as in the reference.  The strip loops of the reference
are written as vectorised slices here; each element sees the same
operations in the same order.  Pinned to fixtures made by the reference's
own FDTD2D (tests/golden/make_golden.py, ``single2d_*``).
"""
from __future__ import annotations

import math

import numpy as np

EPS_0 = 8.854187817e-12
MU_0 = 4.0 * math.pi * 1e-7
C_0 = 299_792_458.0


def cpml_params(n, d, dt, order, sigma_factor, alpha_max, kappa_max):
    """be, ce, bh, ch for one axis (absorbing.py:262-300)."""
    sigma_max = sigma_factor * (order + 1) / (150.0 * math.pi * d)
    out = []
    for shift in (0.0, 0.5):
        rho = (np.arange(n, dtype=np.float64) + shift) / n
        sig = sigma_max * rho ** order
        kap = 1.0 + (kappa_max - 1.0) * rho ** order
        alp = alpha_max * (1.0 - rho)
        b = np.exp(-(sig / kap + alp) * dt / EPS_0)
        c = np.where(np.abs(sig) < 1e-20, 0.0, sig / (sig * kap + kap ** 2 * alp) * (b - 1.0))
        out += [b, c]
    return out  # be, ce, bh, ch


class Single2DOracle:
    """mode "TMZ" (fields ez, hx, hy) or "TEZ" (hz, ex, ey).

    sources: list of (x, y, component, waveform array over steps).
    boundaries: list of ("pec",), ("mur",) or
                ("cpml", thickness, order, sigma_factor, alpha_max, kappa_max).
    """

    def __init__(self, nx, ny, dx, dy, dt, mode, ca, cb, da, db, sources=(), boundaries=(),
                 probe_points=(), record_field=None, record_interval=1):
        self.nx, self.ny, self.dx, self.dy, self.dt, self.mode = nx, ny, dx, dy, dt, mode
        self.ca, self.cb, self.da, self.db = (np.asarray(a, np.float64) for a in (ca, cb, da, db))
        self.sources = list(sources)
        self.boundaries = []
        for b in boundaries:
            if b[0] == "cpml":
                t = int(b[1])
                px = cpml_params(t, dx, dt, *b[2:])
                py = cpml_params(t, dy, dt, *b[2:])
                psi = {k: np.zeros((t, ny)) for k in ("e_xlo", "e_xhi", "h_xlo", "h_xhi")}
                psi.update({k: np.zeros((nx, t)) for k in ("e_ylo", "e_yhi", "h_ylo", "h_yhi")})
                self.boundaries.append(("cpml", t, px, py, psi))
            elif b[0] == "mur":
                self.boundaries.append(("mur", {k: None for k in ("x0", "xn", "y0", "yn")}))
            else:
                self.boundaries.append(("pec",))
        z = lambda: np.zeros((nx, ny))
        if mode == "TMZ":
            self.f = {"Ez": z(), "Hx": z(), "Hy": z()}
        else:
            self.f = {"Hz": z(), "Ex": z(), "Ey": z()}
        self.probe_points = list(probe_points)
        self.record_field = record_field
        self.record_interval = record_interval
        self.probe_data = {pt: [] for pt in self.probe_points}
        self.snapshots = []
        self.n = 0

    # -- field updates (fdtd_2d.py:111-243) --------------------------------------
    def _h(self):
        f, da, db, dx, dy = self.f, self.da, self.db, self.dx, self.dy
        if self.mode == "TMZ":
            ez, hx, hy = f["Ez"], f["Hx"], f["Hy"]
            hx[:, :-1] = da[:, :-1] * hx[:, :-1] - db[:, :-1] / dy * (ez[:, 1:] - ez[:, :-1])
            hy[:-1, :] = da[:-1, :] * hy[:-1, :] + db[:-1, :] / dx * (ez[1:, :] - ez[:-1, :])
        else:
            hz, ex, ey = f["Hz"], f["Ex"], f["Ey"]
            hz[:-1, :-1] = da[:-1, :-1] * hz[:-1, :-1] + db[:-1, :-1] * (
                (ex[:-1, 1:] - ex[:-1, :-1]) / dy - (ey[1:, :-1] - ey[:-1, :-1]) / dx)

    def _e(self):
        f, ca, cb, dx, dy = self.f, self.ca, self.cb, self.dx, self.dy
        if self.mode == "TMZ":
            ez, hx, hy = f["Ez"], f["Hx"], f["Hy"]
            ez[1:, 1:] = ca[1:, 1:] * ez[1:, 1:] + cb[1:, 1:] * (
                (hy[1:, 1:] - hy[:-1, 1:]) / dx - (hx[1:, 1:] - hx[1:, :-1]) / dy)
        else:
            hz, ex, ey = f["Hz"], f["Ex"], f["Ey"]
            ex[:, 1:] = ca[:, 1:] * ex[:, 1:] + cb[:, 1:] / dy * (hz[:, 1:] - hz[:, :-1])
            ey[1:, :] = ca[1:, :] * ey[1:, :] - cb[1:, :] / dx * (hz[1:, :] - hz[:-1, :])

    # -- CPML (absorbing.py:332-561) ---------------------------------------------
    @staticmethod
    def _strips(t, n, interior_edge):
        """Strip index sets: low side cells i (profile t-1-i) and high side
        slots k at cells n-t+k (profile k); H strips stop before the last cell,
        E strips skip cell 0."""
        m = min(t, n - 1) if interior_edge == "h" else min(t, n)
        lo = np.arange(m)
        hi_k = np.arange(m)
        hi_g = n - t + hi_k
        if interior_edge == "h":
            lo_ok = np.ones(m, bool)
            hi_ok = (hi_g >= 0) & (hi_g < n - 1)
        else:
            lo_ok = lo > 0
            hi_ok = (hi_g > 0) & (hi_g < n)
        return lo[lo_ok], hi_k[hi_ok], hi_g[hi_ok]

    def _cpml_h(self, b):
        _, t, px, py, psi = b
        f, dt, dx, dy, nx, ny = self.f, self.dt, self.dx, self.dy, self.nx, self.ny
        _, _, bhx, chx = px
        _, _, bhy, chy = py
        k = dt / MU_0
        lo, hk, hg = self._strips(t, nx, "h")
        loy, hky, hgy = self._strips(t, ny, "h")
        if self.mode == "TMZ":
            ez, hx, hy = f["Ez"], f["Hx"], f["Hy"]
            tgt_x, sgn_x, src_x, tgt_y, sgn_y, src_y = hy, 1.0, ez, hx, -1.0, ez
        else:
            hz, ex, ey = f["Hz"], f["Ex"], f["Ey"]
            tgt_x, sgn_x, src_x, tgt_y, sgn_y, src_y = hz, -1.0, ey, hz, 1.0, ex
        p = psi["h_xlo"]
        p[lo] = bhx[t - 1 - lo][:, None] * p[lo] + chx[t - 1 - lo][:, None] * (src_x[lo + 1] - src_x[lo]) / dx
        tgt_x[lo] += sgn_x * k * p[lo]
        p = psi["h_xhi"]
        p[hk] = bhx[hk][:, None] * p[hk] + chx[hk][:, None] * (src_x[hg + 1] - src_x[hg]) / dx
        tgt_x[hg] += sgn_x * k * p[hk]
        p = psi["h_ylo"]
        p[:, loy] = bhy[t - 1 - loy] * p[:, loy] + chy[t - 1 - loy] * (src_y[:, loy + 1] - src_y[:, loy]) / dy
        tgt_y[:, loy] += sgn_y * k * p[:, loy]
        p = psi["h_yhi"]
        p[:, hky] = bhy[hky] * p[:, hky] + chy[hky] * (src_y[:, hgy + 1] - src_y[:, hgy]) / dy
        tgt_y[:, hgy] += sgn_y * k * p[:, hky]

    def _cpml_e(self, b):
        _, t, px, py, psi = b
        f, dt, dx, dy, nx, ny = self.f, self.dt, self.dx, self.dy, self.nx, self.ny
        bex, cex, _, _ = px
        bey, cey, _, _ = py
        k = dt / EPS_0
        lo, hk, hg = self._strips(t, nx, "e")
        loy, hky, hgy = self._strips(t, ny, "e")

        def xpart(tgt, src, sgn):
            p = psi["e_xlo"]
            p[lo] = bex[t - 1 - lo][:, None] * p[lo] + cex[t - 1 - lo][:, None] * (src[lo] - src[lo - 1]) / dx
            tgt[lo] += sgn * k * p[lo]
            p = psi["e_xhi"]
            p[hk] = bex[hk][:, None] * p[hk] + cex[hk][:, None] * (src[hg] - src[hg - 1]) / dx
            tgt[hg] += sgn * k * p[hk]

        def ypart(tgt, src, sgn):
            p = psi["e_ylo"]
            p[:, loy] = bey[t - 1 - loy] * p[:, loy] + cey[t - 1 - loy] * (src[:, loy] - src[:, loy - 1]) / dy
            tgt[:, loy] += sgn * k * p[:, loy]
            p = psi["e_yhi"]
            p[:, hky] = bey[hky] * p[:, hky] + cey[hky] * (src[:, hgy] - src[:, hgy - 1]) / dy
            tgt[:, hgy] += sgn * k * p[:, hky]

        if self.mode == "TMZ":
            xpart(f["Ez"], f["Hy"], 1.0)
            ypart(f["Ez"], f["Hx"], -1.0)
        else:
            ypart(f["Ex"], f["Hz"], 1.0)
            xpart(f["Ey"], f["Hz"], -1.0)

    def _mur(self, b):
        prev = b[1]
        e = self.f["Ez"] if self.mode == "TMZ" else self.f["Hz"]
        cdt = C_0 * self.dt
        kx = (cdt - self.dx) / (cdt + self.dx)
        ky = (cdt - self.dy) / (cdt + self.dy)
        for key, n in (("x0", self.ny), ("xn", self.ny), ("y0", self.nx), ("yn", self.nx)):
            if prev[key] is None:
                prev[key] = np.zeros(n)
        new = {"x0": e[1, :].copy(), "xn": e[-2, :].copy(), "y0": e[:, 1].copy(), "yn": e[:, -2].copy()}
        e[0, :] = prev["x0"] + kx * (e[1, :] - e[0, :])
        e[-1, :] = prev["xn"] + kx * (e[-2, :] - e[-1, :])
        e[:, 0] = prev["y0"] + ky * (e[:, 1] - e[:, 0])
        e[:, -1] = prev["yn"] + ky * (e[:, -2] - e[:, -1])
        prev.update(new)

    def _pec(self):
        if self.mode == "TMZ":
            ez = self.f["Ez"]
            ez[0, :] = ez[-1, :] = 0.0
            ez[:, 0] = ez[:, -1] = 0.0
        else:
            ex, ey = self.f["Ex"], self.f["Ey"]
            ex[0, :] = ex[-1, :] = 0.0
            ey[:, 0] = ey[:, -1] = 0.0

    # -- one step ------------------------------------------------------------------
    def step(self):
        self._h()
        for b in self.boundaries:
            if b[0] == "cpml":
                self._cpml_h(b)
        self._e()
        for x, y, comp, w in self.sources:   # fdtd_2d.py:245-260
            if comp in (("Ez",) if self.mode == "TMZ" else ("Hz", "Ex", "Ey")):
                self.f[comp][x, y] += w[self.n]
            elif comp in ("Ex", "Ey"):
                raise IndexError("the reference indexes an empty array here")
        for b in self.boundaries:
            if b[0] == "cpml":
                self._cpml_e(b)
            elif b[0] == "mur":
                self._mur(b)
            else:
                self._pec()
        comp = self.record_field or "Ez"
        if self.record_field and self.n % self.record_interval == 0:
            self.snapshots.append(self.f[self.record_field].copy())
        for pt in self.probe_points:
            self.probe_data[pt].append(float(self.f[comp][pt[0], pt[1]]))
        self.n += 1

    def run(self, steps):
        for _ in range(steps):
            self.step()

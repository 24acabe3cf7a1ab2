"""Seeded synthetic surveys for the benchmark and test workloads.

The reference publishes no benchmark data; these generators produce models and
acquisition geometries with the shapes and value ranges of the workloads this
package is measured on.  All positions are the reference's 1-based model
coordinates (sx, gx columns; sz = gz = 1 is the surface row, SWD.m:94-95).
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np


@dataclass
class Survey:
    name: str
    nz: int
    nx: int
    dx: float
    nbc: int
    dt: float
    nt: int
    f0: float
    sx: np.ndarray            # 1-based shot columns
    gx: np.ndarray            # 1-based receiver columns (uniform spacing)
    M: int                    # shot spacing in receivers (SWD.m:96)
    nt_wf: int = 5
    isfs: int = 1
    fd_order: int = 22
    source_type: str = "w"
    # Radon / pick / SoftMax (SWD.m:100-116)
    df: float = 1.0
    fmin: float = 5.0
    fmax: float = 60.0
    vmin: float = 100.0
    vmax: float = 800.0
    dv: float = 2.0
    offset: int = 45
    m: int = 0
    w: int = 3
    ini: int = 10
    soft_arg_norm: float = 1e4
    smooth_z: int = 1
    smooth_x: int = 2
    vs: np.ndarray = field(default=None, repr=False)        # current model
    vs_true: np.ndarray = field(default=None, repr=False)   # model generating the observed data
    vp_ratio: float = 1.73
    # shots of a larger survey (a rank's share): 1-based shot numbers and that survey's shot count
    shot_no: np.ndarray = field(default=None, repr=False)
    ns_total: int = 0

    @property
    def ns(self):
        return int(self.sx.size)

    @property
    def ng(self):
        return int(self.gx.size)

    @property
    def dtx(self):
        return self.dt / self.dx

    @property
    def vp(self):
        return self.vs * self.vp_ratio

    @property
    def vp_true(self):
        return self.vs_true * self.vp_ratio

    @property
    def ds(self):
        """Receiver spacing in metres (SWD.m:97 dg=dg*dx)."""
        return float(self.gx[1] - self.gx[0]) * self.dx

    @property
    def npair(self):
        return int(round(self.fmax / self.df)) - int(round(self.fmin / self.df)) + 1

    @property
    def np_vel(self):
        return int(math.floor((self.vmax - self.vmin) / self.dv + 1e-9)) + 1

    @property
    def nzbc(self):
        return self.nz + (self.fd_order - 20) // 2 + 1 + self.nbc

    @property
    def nxbc(self):
        return self.nx + 2 * self.nbc

    def source(self):
        return ricker(self.f0, self.dt, self.nt)


def ricker(f, dt, nt):
    """Ricker wavelet of core/ricker.m:18-38, zero-padded to nt samples."""
    nw = 2.2 / f / dt
    nw = 2 * math.floor(nw / 2) + 1
    nc = math.floor(nw / 2)
    k = np.arange(1, nw + 1, dtype=np.float64)
    alpha = (nc - k + 1) * f * dt * math.pi
    beta = alpha * alpha
    w0 = (1.0 - beta * 2) * np.exp(-beta)
    if nt < w0.size:
        raise ValueError("nt is smaller than the wavelet length")
    w = np.zeros(nt)
    w[: w0.size] = w0
    return w


def _checker(nz, nx, cell, amp, rng):
    signs = rng.choice([-1.0, 1.0], size=((nz + cell - 1) // cell, (nx + cell - 1) // cell))
    return 1.0 + amp * np.repeat(np.repeat(signs, cell, 0), cell, 1)[:nz, :nx]


def plain_c1(ns=12, nt=6000) -> Survey:
    """30 x 120 grid, dx 0.5 m, 12 shots x 120 receivers, nt 6000 (the CPU-runnable case)."""
    nz, nx = 30, 120
    rng = np.random.default_rng(1)
    base = np.repeat(np.linspace(200.0, 450.0, nz)[:, None], nx, 1)
    vs = base * _checker(nz, nx, 10, 0.10, rng)
    vs_true = vs.copy()
    zc, xc = nz // 2, nx // 2
    zz, xx = np.mgrid[0:nz, 0:nx]
    vs_true *= 1.0 + 0.10 * np.exp(-(((zz - zc) / 6.0) ** 2 + ((xx - xc) / 12.0) ** 2))
    sx = np.arange(1, 112, 10)[:ns]
    return Survey("plain-30x120", nz, nx, 0.5, 20, 1e-4, nt, 30.0, sx, np.arange(1, nx + 1), 10,
                  vs=vs, vs_true=vs_true)


def batched_c2(ns=96, nt=8000) -> Survey:
    """100 x 600 grid, dx 0.5 m, 96 shots x 600 receivers, nt 8000."""
    nz, nx = 100, 600
    rng = np.random.default_rng(2)
    d1 = int(rng.integers(20, 35))
    d2 = int(rng.integers(55, 75))
    vs = np.empty((nz, nx))
    vs[:d1] = 180.0
    vs[d1:d2] = 320.0
    vs[d2:] = 500.0
    zz, xx = np.mgrid[0:nz, 0:nx]
    r = 8.0 / 0.5
    zc, xc = int(rng.integers(20, 60)), int(rng.integers(150, 450))
    vs_true = vs * (1.0 - 0.15 * np.exp(-(((zz - zc) ** 2 + (xx - xc) ** 2) / (r * r))))
    sx = (1 + 6 * np.arange(96))[:ns]
    return Survey("batched-100x600", nz, nx, 0.5, 30, 5e-5, nt, 25.0, sx, np.arange(1, nx + 1), 6,
                  vs=vs, vs_true=vs_true)


def tiny(nz=8, nx=24, nbc=6, nt=400, ns=3, seed=3) -> Survey:
    """A small grid for quick parity checks."""
    rng = np.random.default_rng(seed)
    vs = 200.0 + 150.0 * rng.random((nz, nx))
    sx = 1 + 4 * np.arange(ns)
    s = Survey(f"tiny-{nz}x{nx}", nz, nx, 0.5, nbc, 1e-4, nt, 60.0, sx, np.arange(1, nx + 1), 4,
               vs=vs, vs_true=vs * 1.05, offset=12, fmin=40.0, fmax=200.0, df=25.0, vmin=100.0, vmax=800.0,
               dv=5.0, ini=3)
    return s


def served_surveys(n=16, seed=4):
    """Surveys of the served request stream: grids log-uniform from 60 x 200 to 300 x 1200
    (dx 0.5 m), 8-64 shots spread along the line with an integer spacing, nt 3000-10000 in
    steps of 50, seeded random layered Vs (150-600 m/s) with a +/-5% checkerboard."""
    rng = np.random.default_rng(seed)
    out = []
    for k in range(n):
        nz = int(round(math.exp(rng.uniform(math.log(60), math.log(300)))))
        nx = int(round(math.exp(rng.uniform(math.log(200), math.log(1200)))))
        ns = int(rng.integers(8, 65))
        M = max(1, (nx - 1) // ns)
        nt = int(round(rng.uniform(3000, 10000) / 50)) * 50
        nl = int(rng.integers(3, 7))
        cuts = np.sort(rng.choice(np.arange(1, nz), nl - 1, replace=False))
        vel = np.sort(rng.uniform(150.0, 600.0, nl))
        vs = np.repeat(vel[np.searchsorted(cuts, np.arange(nz), side="right")][:, None], nx, 1)
        vs = vs * _checker(nz, nx, 10, 0.05, rng)
        sx = 1 + M * np.arange(ns)
        out.append(Survey(f"served-{k}-{nz}x{nx}", nz, nx, 0.5, 30, 5e-5, nt, 25.0, sx, np.arange(1, nx + 1), M,
                          vs=vs, vs_true=vs * 1.02))
    return out


def served_stream(n_requests=64, n_surveys=16, rate=2.0, seed=4):
    """(arrival time s, survey index, kind, model scale) of a Poisson request stream over the
    served surveys: half gradients, half line-search misfits, each on a slightly scaled model."""
    rng = np.random.default_rng(seed + 1)
    t = np.cumsum(rng.exponential(1.0 / rate, n_requests))
    idx = rng.integers(0, n_surveys, n_requests)
    kind = np.where(rng.random(n_requests) < 0.5, "gradient", "misfit")
    scale = 1.0 + rng.uniform(-0.02, 0.02, n_requests)
    return list(zip(t.tolist(), idx.tolist(), kind.tolist(), scale.tolist()))


def smooth_curve(s, seed=0):
    """A synthetic observed dispersion curve per shot (npair x ns): a decreasing phase velocity
    inside the Radon axis, standing in for picks of observed data."""
    rng = np.random.default_rng(seed)
    f = np.arange(s.npair)[:, None]
    span = s.vmax - s.vmin
    base = s.vmin + span * (0.15 + 0.35 * np.exp(-f / max(1.0, s.npair / 3)))
    return np.round(base + rng.normal(0, 2.0, (1, s.ns)))


def _grf(shape, corr, rng):
    """Zero-mean, unit-variance Gaussian random field with a Gaussian correlation of `corr` cells."""
    nz, nx = shape
    w = rng.standard_normal(shape)
    kz = np.fft.fftfreq(nz)[:, None]
    kx = np.fft.rfftfreq(nx)[None, :]
    f = np.fft.irfft2(np.fft.rfft2(w) * np.exp(-2 * (np.pi * corr) ** 2 * (kz ** 2 + kx ** 2)), s=shape)
    return (f - f.mean()) / f.std()


def large_c5(ns=240, nt=20000) -> Survey:
    """400 x 3000 grid, dx 0.25 m, 240 shots (every 10th column) x 1200 receivers (every 2nd), nt 20000,
    dt 2.5e-5 s, Ricker f0 40 Hz.  Vs: seeded layers from 150 to 800 m/s whose interfaces drop
    3 m across a vertical fault, times a Gaussian random field (correlation 5 m, +/-8% at two
    standard deviations); Vp = 1.8 Vs."""
    nz, nx, dx = 400, 3000, 0.25
    rng = np.random.default_rng(5)
    nl = 6
    vel = np.linspace(150.0, 800.0, nl)
    cuts = np.sort(rng.choice(np.arange(30, nz - 30), nl - 1, replace=False))
    throw = int(round(3.0 / dx))
    xf = int(rng.integers(nx // 3, 2 * nx // 3))
    z = np.arange(nz)[:, None]
    left = np.searchsorted(cuts, z, side="right")
    right = np.searchsorted(cuts + throw, z, side="right")
    layer = np.where(np.arange(nx)[None, :] < xf, left, right)
    vs = vel[layer] * (1.0 + 0.04 * _grf((nz, nx), 5.0 / dx, rng))
    vs_true = vs.copy()
    zz, xx = np.mgrid[0:nz, 0:nx]
    vs_true *= 1.0 - 0.10 * np.exp(-(((zz - nz // 3) / 40.0) ** 2 + ((xx - nx // 2) / 200.0) ** 2))
    # shots every 10 columns (5 receivers): 240 shots then span the 2400 columns the receivers
    # cover (a 12-column spacing would put the last 40 shots' windows past the receiver line)
    sx = 1 + 10 * np.arange(ns)
    return Survey("large-400x3000", nz, nx, dx, 40, 2.5e-5, nt, 40.0, sx, np.arange(1, 2400, 2), 5,
                  vs=vs, vs_true=vs_true, vp_ratio=1.8)

"""Seeded synthetic disk densities for the pot3 workloads.

There is no public benchmark or dataset for this path; the reference's own
inputs (hscf models read as fort.2, radhydro/io.f:157-183) need a Fortran
build.  These generators produce self-gravitating flared-disk densities with
the shapes, sizes and value ranges of the reference's runs:

* grid: ROF3N = 1/JMAX, ZOF3N = 0.5/KMAX, R(J) = (J-2)*ROF3N, RHF = R + ROF3N/2
  (radhydro/io.f:194-203), azimuth psi = (L - 1/2)*DTHETA (pot/boundary.f:32);
* base disk: Sigma(r) = (r/r_out)^s * exp(-(r/(0.8 r_out))^4), H = h*r,
  rho = Sigma/(sqrt(2 pi) H) * exp(-z^2 / 2H^2), r_out = R(JMAX+1);
* multiplicative perturbations: cell noise (1 + 1e-3 u), u ~ U(-1,1) drawn in
  Fortran order; an m=2 log spiral of amplitude 0.05 and pitch 15 degrees; a
  random m<=32 spectrum with amplitudes 0.02 m^-2;
* floor rho >= 1e-10 max(rho) (radhydro/io.f:178-180).

Arrays are RHO(JMAX2, KMAX2, LMAX) in Fortran (column-major) order.
"""
from __future__ import annotations

import math
from dataclasses import dataclass

import numpy as np

PI = 3.1415926535897932


@dataclass
class Grid:
    jmax: int
    kmax: int
    lmax: int
    delr: float
    delz: float

    @property
    def dtheta(self) -> float:
        return 2.0 * PI / float(self.lmax)

    def r(self):
        j = np.arange(1, self.jmax + 3, dtype=np.float64)
        return (j - 2.0) * self.delr

    def rhf(self):
        return self.r() + self.delr / 2.0

    def z(self):
        k = np.arange(1, self.kmax + 3, dtype=np.float64)
        return (k - 2.0) * self.delz

    def zhf(self):
        return self.z() + self.delz / 2.0


def default_grid(jmax: int, kmax: int, lmax: int) -> Grid:
    return Grid(jmax, kmax, lmax, 1.0 / jmax, 0.5 / kmax)


def disk_density(jmax: int, kmax: int, lmax: int, seed: int, *, slope: float = -1.5,
                 h: float = 0.05, spiral: bool = False, spectrum: bool = False,
                 noise: float = 1e-3, rng: np.random.Generator | None = None) -> np.ndarray:
    """RHO(JMAX2,KMAX2,LMAX) float64, Fortran order, zero outside j,k = 2..max+1."""
    g = default_grid(jmax, kmax, lmax)
    if rng is None:
        rng = np.random.default_rng(seed)
    rhf = g.rhf()[1:jmax + 1]          # j = 2..JMAX+1
    zhf = g.zhf()[1:kmax + 1]          # k = 2..KMAX+1
    r_out = g.r()[jmax]                # R(JMAX+1)
    psi = (np.arange(1, lmax + 1, dtype=np.float64) - 0.5) * g.dtheta
    sig = (rhf / r_out) ** slope * np.exp(-(rhf / (0.8 * r_out)) ** 4)
    H = h * rhf
    base = (sig / (math.sqrt(2.0 * PI) * H))[:, None] * np.exp(-(zhf[None, :] ** 2) / (2.0 * H[:, None] ** 2))
    # cell noise drawn with j fastest, then k, then l
    u = rng.uniform(-1.0, 1.0, size=(lmax, kmax, jmax))
    rho = base[:, :, None] * (1.0 + noise * np.transpose(u, (2, 1, 0)))
    if spiral:
        pitch = math.tan(math.radians(15.0))
        arg = 2.0 * (psi[None, :] - np.log(rhf / r_out)[:, None] / pitch)
        rho *= (1.0 + 0.05 * np.cos(arg))[:, None, :]
    if spectrum:
        phases = rng.uniform(0.0, 2.0 * PI, size=32)
        m = np.arange(1, 33, dtype=np.float64)
        pert = 1.0 + np.sum(0.02 * m[:, None] ** -2 * np.cos(m[:, None] * psi[None, :] + phases[:, None]), axis=0)
        rho *= pert[None, None, :]
    rho = np.maximum(rho, 1e-10 * rho.max())
    out = np.zeros((jmax + 2, kmax + 2, lmax), dtype=np.float64, order="F")
    out[1:jmax + 1, 1:kmax + 1, :] = rho
    return out


def config_density(config: int, index: int = 0) -> tuple[np.ndarray, Grid]:
    """The seeded inputs of the five pot3 workloads.

    1: 64x32x64 base disk + noise (seed 1)
    2: 256x128x256 + m=2 spiral (seed 2)
    3: 256x128x256 + spiral + m<=32 spectrum (seed 3)
    4: batch member `index` (seed 1000+index): JMAX in {64,128,256}, KMAX in
       {32,64,128}, LMAX in {64,128,256}, slope ~ U[-2,-1], h ~ U[0.03,0.1]
    5: serving request `index` (seed 10**6+index): 20% 512x128x512, else the
       config-4 size set.
    """
    if config == 1:
        return disk_density(64, 32, 64, 1), default_grid(64, 32, 64)
    if config == 2:
        return disk_density(256, 128, 256, 2, spiral=True), default_grid(256, 128, 256)
    if config == 3:
        return disk_density(256, 128, 256, 3, spiral=True, spectrum=True), default_grid(256, 128, 256)
    if config in (4, 5):
        seed = (1000 if config == 4 else 10**6) + index
        rng = np.random.default_rng(seed)
        if config == 5 and rng.uniform() < 0.2:
            J, K, L = 512, 128, 512
        else:
            J = int(rng.choice([64, 128, 256]))
            K = int(rng.choice([32, 64, 128]))
            L = int(rng.choice([64, 128, 256]))
        slope = float(rng.uniform(-2.0, -1.0))
        h = float(rng.uniform(0.03, 0.1))
        rho = disk_density(J, K, L, seed, slope=slope, h=h, spiral=True, spectrum=True, rng=rng)
        return rho, default_grid(J, K, L)
    raise ValueError(f"unknown config {config}")

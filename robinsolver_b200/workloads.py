"""Seeded synthetic Helmholtz workloads (potential, point sources, plane waves).

The benchmark problems are 2D boxes [0,1]^2 with a smooth random potential

    k(x) = kb * (1 + 0.3 * sum_j a_j * exp(-|x - c_j|^2 / (2 w^2))) + i * delta * kb,

bump centres c_j ~ U([0.2, 0.8]^2), amplitudes a_j ~ U(-1, 1), width w = 0.08, and
an impedance boundary condition u_n - i*kb*u = g.  Right-hand sides are either a
Gaussian point source f = exp(-|x - x0|^2 / (2 * 0.05^2)), x0 ~ U([0.1, 0.9]^2),
with g = 0, or a plane wave exp(i*kb*d.x), d = (cos t, sin t), t ~ U(0, 2 pi), fed
through g = (d_n - i*kb) exp(i*kb*d.x) = i*kb*(d.n - 1) exp(i*kb*d.x) with f = 0.

Draw order is fixed: bump centres, amplitudes, then one draw per right-hand side.
The reference's FD boundary row is ``u_n + i*opts%kb*u`` (fd_module.f90:131), so
the impedance condition u_n - i*kb*u is expressed with ``opts.kb = -kb`` and
``bndry_params = [[i*opts.kb, 1], [-i*opts.kb, 1]]`` (the choice of example.f90:64-65),
which gives zeta = 0 and nu = -1 in the merge.

Callbacks are vectorised: they take an ``(npts, 3)`` array of points.  Face
callbacks take face-local coordinates (x faces: y in column 0; y faces: x in column 0),
the coordinates the reference hands to ``g_face`` (fd_module.f90:648-651).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

# (N, L, kb, nbumps, delta, nrhs) per benchmark configuration
CONFIGS = {
    1: dict(N=64, L=4, kb=20.0, nbumps=5, delta=0.01, nrhs=1, kinds="point"),
    2: dict(N=512, L=10, kb=100.0, nbumps=40, delta=0.005, nrhs=16, kinds="alternate"),
    4: dict(N=1024, L=12, kb=200.0, nbumps=100, delta=0.002, nrhs=32, kinds="plane"),
}


@dataclass
class Potential:
    """k(x) = kb^p (1 + 0.3 sum_j a_j bump_j(x)) + i delta kb^p.  p = 1 is the formula used
    literally as ``ell_op%k`` (fd_module.f90:145 adds k itself, not its square); p = 2 is the
    oscillatory stress variant whose coefficient is a squared wavenumber, kb^2 (1 + ...)."""
    kb: float
    delta: float
    centres: np.ndarray
    amps: np.ndarray
    width: float = 0.08
    power: int = 1

    def __call__(self, X):
        X = np.asarray(X, dtype=np.float64)
        s = np.zeros(X.shape[0])
        w2 = 2.0 * self.width * self.width
        for c, a in zip(self.centres, self.amps):
            r2 = (X[:, 0] - c[0]) ** 2 + (X[:, 1] - c[1]) ** 2
            s += a * np.exp(-r2 / w2)
        scale = self.kb ** self.power
        return scale * (1.0 + 0.3 * s) + 1j * (self.delta * scale)


@dataclass
class PointSource:
    x0: np.ndarray
    width: float = 0.05

    def __call__(self, X):
        X = np.asarray(X, dtype=np.float64)
        r2 = (X[:, 0] - self.x0[0]) ** 2 + (X[:, 1] - self.x0[1]) ** 2
        return np.exp(-r2 / (2.0 * self.width * self.width)) + 0j


def zero_fun(X):
    return np.zeros(np.asarray(X).shape[0], dtype=np.complex128)


@dataclass
class PlaneWaveFace:
    """g on one face of the box for the plane wave exp(i*kb*d.x)."""
    kb: float
    d: np.ndarray
    face: int                  # 1..4 = x1 x2 y1 y2
    domain: np.ndarray         # (2,3)

    def __call__(self, X):
        X = np.asarray(X, dtype=np.float64)
        t = X[:, 0]
        if self.face in (1, 2):
            x = np.full_like(t, self.domain[self.face - 1, 0])
            y = t
            n = np.array([-1.0, 0.0]) if self.face == 1 else np.array([1.0, 0.0])
        else:
            x = t
            y = np.full_like(t, self.domain[self.face - 3, 1])
            n = np.array([0.0, -1.0]) if self.face == 3 else np.array([0.0, 1.0])
        dn = self.d[0] * n[0] + self.d[1] * n[1]
        e = np.exp(1j * self.kb * (self.d[0] * x + self.d[1] * y))
        return 1j * self.kb * (dn - 1.0) * e


@dataclass
class RHS:
    kind: str
    f: object
    g: list


@dataclass
class Workload:
    N: int
    L: int
    kb: float
    domain: np.ndarray
    potential: Potential
    rhs: list = field(default_factory=list)

    @property
    def h_tgt(self):
        return 1.0 / self.N

    @property
    def opts_kb(self):
        return -self.kb

    @property
    def bndry_params(self):
        k = self.opts_kb
        return np.array([[1j * k, 1.0], [-1j * k, 1.0]], dtype=np.complex128)


def make_workload(config_id: int, instance: int = 0, nrhs: int | None = None, N=None, L=None,
                  kb=None, nbumps=None, delta=None, kinds=None, kpower: int = 1) -> Workload:
    """Seeded workload; seed = 1000 * config_id + instance.  Keyword overrides allow
    smaller variants with the same generator; ``kpower=2`` gives the squared-wavenumber
    potential kb^2 (1 + ...) with the same draws."""
    c = dict(CONFIGS[config_id])
    for k_, v in dict(N=N, L=L, kb=kb, nbumps=nbumps, delta=delta, nrhs=nrhs, kinds=kinds).items():
        if v is not None:
            c[k_] = v
    rng = np.random.default_rng(1000 * config_id + instance)
    centres = rng.uniform(0.2, 0.8, size=(c["nbumps"], 2))
    amps = rng.uniform(-1.0, 1.0, size=c["nbumps"])
    dom = np.array([[0.0, 0.0, 0.0], [1.0, 1.0, 1.0]])
    pot = Potential(kb=c["kb"], delta=c["delta"], centres=centres, amps=amps, power=kpower)
    wl = Workload(N=c["N"], L=c["L"], kb=c["kb"], domain=dom, potential=pot)
    for r in range(c["nrhs"]):
        kind = c["kinds"]
        if kind == "alternate":
            kind = "point" if r % 2 == 0 else "plane"
        if kind == "point":
            x0 = rng.uniform(0.1, 0.9, size=2)
            wl.rhs.append(RHS("point", PointSource(x0), [zero_fun] * 4))
        else:
            th = rng.uniform(0.0, 2.0 * np.pi)
            d = np.array([np.cos(th), np.sin(th)])
            wl.rhs.append(RHS("plane", zero_fun,
                              [PlaneWaveFace(c["kb"], d, f, dom) for f in range(1, 5)]))
    return wl

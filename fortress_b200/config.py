"""Run configuration: the positional records of INPUT/input{1,2,3}D.dat and
the quantities the reference derives from them.

Record order follows cgpe1d.f90:233-260 (1D), cgpe2d.f90:234-261 (2D) and
cgpe3d.f90:239-266 (3D); README.md:53-86 documents the file.  Fortran
list-directed reads take the first values of each record and ignore the rest
of the line (the "#..." comments), accept ',' or blanks as separators and 'D'
exponents.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field

# cgpe1d.f90:33-37
PI = 4.0 * math.atan(1.0)
AMU = 1.66e-27
HBAR = 1.054560653e-34
AU = 0.529177208e-10
EPS = 1.0e-40
TOL_NR = 1.0e-6

_NUM = re.compile(r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eEdD][-+]?\d+)?")


def simpson_weights(n, dx):
    """Node weights of simpson.f90:4-21 (composite 1/3 rule on 1..N-3 plus a
    3/8 rule on N-3..N), obtained by applying the routine to unit vectors."""
    import numpy as np
    w = np.zeros(n)
    for t in range(n):
        f = np.zeros(n)
        f[t] = 1.0
        f1 = f[1] + f[n - 5]
        f2 = f[2]
        for i in range(4, n - 5, 2):
            f1 += f[i - 1]
            f2 += f[i]
        w[t] = dx * (f[0] + 4.0 * f1 + 2.0 * f2 + f[n - 4]) / 3.0 + 3.0 * dx * (f[n - 4] + 3.0 * (f[n - 3] + f[n - 2]) + f[n - 1]) / 8.0
    return w


class InputError(ValueError):
    pass


def _record(line):
    body = line.split("#", 1)[0]
    return [t.replace("D", "E").replace("d", "e") for t in _NUM.findall(body)]


@dataclass
class RunConfig:
    dim: int
    spin: int = 1
    niter: int = 0
    stp: int = 1
    nstp: int = 1
    threads: int = 1
    n: tuple = (1, 1, 1)
    d: tuple = (1.0, 1.0, 1.0)
    dt: float = 0.0
    mass: float = 0.0
    a: tuple = (0.0, 0.0, 0.0)
    natoms: int = 0
    nu: tuple = (1.0, 1.0, 1.0)
    tol: float = 0.0
    switch_im: int = 1
    gamma: tuple = (0.0, 0.0, 0.0)
    option_fpc: int = 4
    mag: float = 0.0
    switch_soc: int = 0
    extra: dict = field(default_factory=dict)

    # ------------------------------------------------------------ parsing
    @classmethod
    def from_text(cls, text: str, dim: int) -> "RunConfig":
        lines = [ln for ln in text.splitlines()]
        pos = [0]

        def take(k, kind=float):
            """Read the next record with at least k values (list-directed
            reads continue onto following records when one is short)."""
            vals = []
            while len(vals) < k:
                if pos[0] >= len(lines):
                    raise InputError("input file ended early")
                vals += _record(lines[pos[0]])
                pos[0] += 1
            return [kind(float(v)) if kind is int else kind(v) for v in vals[:k]]

        def skip():
            if pos[0] < len(lines):
                pos[0] += 1

        c = cls(dim=dim)
        c.spin = take(1, int)[0]
        if c.spin not in (1, 2):
            raise InputError("SPIN must be 1 or 2")
        c.niter = take(1, int)[0]
        c.stp, c.nstp = take(2, int)
        c.threads = take(1, int)[0]
        c.n = tuple(take(dim, int) + [1] * (3 - dim))
        v = take(dim + 1, float)
        c.d = tuple(v[:dim] + [1.0] * (3 - dim))
        c.dt = v[dim]
        c.mass = take(1, float)[0]
        v = take(2 if c.spin == 1 else 3, float)
        c.a = tuple(v + [0.0] * (3 - len(v)))
        c.natoms = take(1, int)[0]
        c.nu = tuple(take(3, float))
        c.tol = take(1, float)[0]
        c.switch_im = take(1, int)[0]
        g = take(dim, float)
        c.gamma = tuple(g + [0.0] * (3 - dim))
        # cgpe1d.f90:250, cgpe2d.f90:251, cgpe3d.f90:256
        c.switch_soc = int(any(abs(x) > EPS for x in g))
        if c.switch_soc == 0:
            c.option_fpc = take(1, int)[0]
        else:
            skip()
        if c.switch_im == 1 and c.switch_soc == 0:
            c.mag = take(1, float)[0]
        else:
            skip()
        return c

    @classmethod
    def from_file(cls, path: str, dim: int) -> "RunConfig":
        with open(path) as f:
            return cls.from_text(f.read(), dim)

    # ---------------------------------------------------------- derived
    @property
    def ms(self):
        return 2 * self.spin + 1

    @property
    def alpha(self):
        nux, nuy, nuz = self.nu
        return (nux / nux, nuy / nux, nuz / nux)     # cgpe1d.f90:267-269

    @property
    def aosc(self):
        omegam = 2.0 * PI * self.nu[0]                # cgpe1d.f90:321-322
        return math.sqrt(HBAR / (self.mass * AMU * omegam))

    def tau(self):
        """TAU(0:2) (cgpe1d.f90:324-332, cgpe2d.f90:328-336,
        cgpe3d.f90:337-345): the dimensionless couplings with the reference's
        factor 2 and the q1D/q2D geometric factor."""
        _, ay, az = self.alpha
        if self.dim == 1:
            geo = math.sqrt(ay * az) / (2.0 * PI)
        elif self.dim == 2:
            geo = math.sqrt(az / (2.0 * PI))
        else:
            geo = 1.0
        a0, a2, a4 = (x * AU for x in self.a)
        aosc = self.aosc
        if self.spin == 1:
            n = float(__import__("numpy").float32(self.natoms))   # REAL(NATOMS)
            t0 = 2.0 * geo * (4.0 * PI * n * (a0 + 2.0 * a2) / (3.0 * aosc))
            t1 = 2.0 * geo * (4.0 * PI * n * (a2 - a0) / (3.0 * aosc))
            return (t0, t1, 0.0)
        n = float(self.natoms)
        t0 = 2.0 * (geo * 4.0 * PI * n * (4.0 * a2 + 3.0 * a4) / (7.0 * aosc))
        t1 = 2.0 * (geo * 4.0 * PI * n * (a4 - a2) / (7.0 * aosc))
        t2 = 2.0 * (geo * 4.0 * PI * n * (7.0 * a0 - 10.0 * a2 + 3.0 * a4) / (7.0 * aosc))
        return (t0, t1, t2)

    def params(self, precision="fp64"):
        """Keyword arguments for :class:`fortress_b200.Propagator`."""
        return dict(dim=self.dim, spin=self.spin, n=self.n[: self.dim], d=self.d[: self.dim],
                    dt=self.dt, imag_time=bool(self.switch_im), tau=self.tau(),
                    gamma=self.gamma[: self.dim], alpha=self.alpha, precision=precision, mag=self.mag)

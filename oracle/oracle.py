"""Python face of the CPU oracle (test infrastructure only).

Only tests/, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` import this module, and only to compare results against.  The
product package ``fortress_b200`` never imports it.

It wraps ``libcgpe_oracle.so`` (``cgpe_oracle.c``, the FP64 restatement of the
FORTRESS operators) and restates, in Python, the reference's main loop
(SRC/cgpe1d.f90:433-519, cgpe2d.f90:440-531, cgpe3d.f90:451-567): split step,
NORMC every step, NORMT in imaginary time, ENERGY/RAD/CONV every STP steps,
exit on CONV <= TOL or CONV_EN <= TOL before the file2/file3 rows are written.
"""
from __future__ import annotations

import ctypes
import os
import re
import subprocess
from dataclasses import dataclass, field

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def build():
    """Compile libcgpe_oracle.so with the Makefile beside this file."""
    env = dict(os.environ)
    env.pop("CC", None)
    subprocess.run(["make", "-s", "-C", _HERE], check=True, env=env)


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(_HERE, "libcgpe_oracle.so")
        src = os.path.join(_HERE, "cgpe_oracle.c")
        if not os.path.exists(path) or os.path.getmtime(path) < os.path.getmtime(src):
            build()
        L = ctypes.CDLL(path)
        P = ctypes.POINTER(ctypes.c_double)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_void_p]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        for n in ("orc_set_state", "orc_get_state"):
            getattr(L, n).argtypes = [ctypes.c_void_p, P]
        L.orc_grids.argtypes = [ctypes.c_void_p] + [P] * 6
        for n in ("orc_fft", "orc_bft", "orc_ke", "orc_soc", "orc_se", "orc_sp"):
            getattr(L, n).argtypes = [ctypes.c_void_p]
        L.orc_fft1d.argtypes = [ctypes.c_int, P, ctypes.c_int]
        L.orc_expm_se2.argtypes = [P, ctypes.c_double, ctypes.c_double, P]
        L.orc_simpson.restype = ctypes.c_double
        L.orc_simpson.argtypes = [P, ctypes.c_int, ctypes.c_double]
        L.orc_diff.argtypes = [P, ctypes.c_int, ctypes.c_double, P]
        L.orc_normc.argtypes = [ctypes.c_void_p, P]
        L.orc_normt.restype = ctypes.c_double
        L.orc_normt.argtypes = [ctypes.c_void_p]
        L.orc_rad.argtypes = [ctypes.c_void_p, P]
        L.orc_energy.argtypes = [ctypes.c_void_p, P, P, P]
        L.orc_step.argtypes = [ctypes.c_void_p, ctypes.c_int, P]
        L.orc_step.restype = ctypes.c_int
        L.orc_set_mag.argtypes = [ctypes.c_void_p, ctypes.c_double]
        L.orc_get_sig.argtypes = [ctypes.c_void_p, P]
        L.orc_maxdiff.restype = ctypes.c_double
        L.orc_maxdiff.argtypes = [ctypes.c_void_p, P]
        L.orc_initialize.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.orc_tau.argtypes = ([ctypes.c_int, ctypes.c_int, ctypes.c_int] + [ctypes.c_double] * 7 + [P, P])
        L.orc_num_threads.restype = ctypes.c_int
        L.orc_set_num_threads.argtypes = [ctypes.c_int]
        _LIB = L
    return _LIB


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


class _Params(ctypes.Structure):
    _fields_ = [("dim", ctypes.c_int), ("spin", ctypes.c_int),
                ("nx", ctypes.c_int), ("ny", ctypes.c_int), ("nz", ctypes.c_int),
                ("dx", ctypes.c_double), ("dy", ctypes.c_double), ("dz", ctypes.c_double),
                ("dt", ctypes.c_double), ("imag", ctypes.c_int),
                ("tau", ctypes.c_double * 3),
                ("gx", ctypes.c_double), ("gy", ctypes.c_double), ("gz", ctypes.c_double),
                ("ax", ctypes.c_double), ("ay", ctypes.c_double), ("az", ctypes.c_double)]


# ----------------------------------------------------------------- inputs
_NUM = re.compile(r"[-+]?(?:\d+\.?\d*|\.\d+)(?:[eEdD][-+]?\d+)?")


def _values(line):
    body = line.split("#", 1)[0]
    return [float(t.replace("D", "E").replace("d", "e")) for t in _NUM.findall(body)]


@dataclass
class Input:
    """The positional records of INPUT/input{1,2,3}D.dat (README.md:53-86),
    read in the order of cgpe1d.f90:233-260 / cgpe2d.f90:234-261 /
    cgpe3d.f90:239-266."""
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

    @classmethod
    def parse(cls, text, dim):
        recs = [ln for ln in text.splitlines() if ln.strip()]
        it = iter(recs)
        nxt = lambda: _values(next(it))
        s = cls(dim=dim)
        s.spin = int(nxt()[0])
        s.niter = int(nxt()[0])
        v = nxt(); s.stp, s.nstp = int(v[0]), int(v[1])
        s.threads = int(nxt()[0])
        v = nxt(); n = [int(x) for x in v[:dim]] + [1] * (3 - dim); s.n = tuple(n)
        v = nxt(); s.d = tuple(list(v[:dim]) + [1.0] * (3 - dim)); s.dt = v[dim]
        s.mass = nxt()[0]
        v = nxt(); s.a = (v[0], v[1], v[2] if s.spin == 2 else 0.0)
        s.natoms = int(nxt()[0])
        v = nxt(); s.nu = (v[0], v[1], v[2])
        s.tol = nxt()[0]
        s.switch_im = int(nxt()[0])
        v = nxt(); g = list(v[:dim]) + [0.0] * (3 - dim); s.gamma = tuple(g)
        s.switch_soc = int(any(abs(x) > 1e-40 for x in g))
        v = nxt()
        if s.switch_soc == 0 and v:
            s.option_fpc = int(v[0])
        v = nxt() if True else []
        if s.switch_im == 1 and s.switch_soc == 0 and v:
            s.mag = v[0]
        return s

    @property
    def alpha(self):
        nux, nuy, nuz = self.nu
        return (nux / nux, nuy / nux, nuz / nux)

    def tau(self):
        t = np.zeros(3)
        aosc = np.zeros(1)
        lib().orc_tau(self.dim, self.spin, self.natoms, self.mass, self.a[0], self.a[1], self.a[2],
                      self.nu[0], self.nu[1], self.nu[2], _dp(t), _dp(aosc))
        return t, float(aosc[0])


def params_from_input(inp: Input, tau=None):
    t = inp.tau()[0] if tau is None else np.asarray(tau, float)
    return dict(dim=inp.dim, spin=inp.spin, nx=inp.n[0], ny=inp.n[1], nz=inp.n[2],
                dx=inp.d[0], dy=inp.d[1], dz=inp.d[2], dt=inp.dt, imag=inp.switch_im,
                tau=tuple(t), gx=inp.gamma[0], gy=inp.gamma[1], gz=inp.gamma[2],
                ax=inp.alpha[0], ay=inp.alpha[1], az=inp.alpha[2])


# ------------------------------------------------------------------ handle
class Oracle:
    """One CPU propagator instance (state PHI(NX,NY,NZ,M) complex128,
    Fortran order)."""

    def __init__(self, **kw):
        p = _Params()
        p.dim = kw["dim"]; p.spin = kw["spin"]
        p.nx = kw["nx"]; p.ny = kw.get("ny", 1); p.nz = kw.get("nz", 1)
        p.dx = kw["dx"]; p.dy = kw.get("dy", 1.0); p.dz = kw.get("dz", 1.0); p.dt = kw["dt"]
        p.imag = int(kw["imag"])
        for i, v in enumerate(kw["tau"]):
            p.tau[i] = v
        p.gx = kw.get("gx", 0.0); p.gy = kw.get("gy", 0.0); p.gz = kw.get("gz", 0.0)
        p.ax = kw.get("ax", 1.0); p.ay = kw.get("ay", 1.0); p.az = kw.get("az", 1.0)
        self.kw = dict(kw)
        self.dim, self.spin, self.ms = p.dim, p.spin, 2 * p.spin + 1
        self.shape = (p.nx, p.ny if p.dim >= 2 else 1, p.nz if p.dim >= 3 else 1)
        self._p = p
        self.h = lib().orc_create(ctypes.byref(p))

    def __del__(self):
        h = getattr(self, "h", None)
        if h:
            lib().orc_destroy(h)
            self.h = None

    @property
    def npts(self):
        return int(np.prod(self.shape))

    def set_state(self, phi):
        a = np.asfortranarray(np.asarray(phi, np.complex128).reshape(self.shape + (self.ms,), order="F"))
        flat = np.ascontiguousarray(a.reshape(-1, order="F"))
        lib().orc_set_state(self.h, _dp(flat.view(np.float64)))

    def state(self):
        flat = np.empty(self.npts * self.ms, np.complex128)
        lib().orc_get_state(self.h, _dp(flat.view(np.float64)))
        return flat.reshape(self.shape + (self.ms,), order="F")

    def grids(self):
        nx, ny, nz = self.shape
        arrs = [np.empty(n) for n in (nx, ny, nz, nx, ny, nz)]
        lib().orc_grids(self.h, *[_dp(a) for a in arrs])
        return arrs

    def initialize(self, option_fpc=4, mag=0.0):
        lib().orc_initialize(self.h, option_fpc, mag)

    # operators in the reference order
    def fft(self): lib().orc_fft(self.h)
    def bft(self): lib().orc_bft(self.h)
    def ke(self): lib().orc_ke(self.h)
    def soc(self): lib().orc_soc(self.h)
    def se(self): lib().orc_se(self.h)
    def sp(self): lib().orc_sp(self.h)

    def normc(self):
        n = np.zeros(self.ms); lib().orc_normc(self.h, _dp(n)); return n

    def normt(self):
        return lib().orc_normt(self.h)

    def rad(self):
        r = np.zeros(self.ms); lib().orc_rad(self.h, _dp(r)); return r

    def energy(self):
        mu = np.zeros(self.ms); en = np.zeros(1); mz = np.zeros(1)
        lib().orc_energy(self.h, _dp(mu), _dp(en), _dp(mz))
        return float(en[0]), mu, float(mz[0])

    def step(self, n=1):
        norm = np.zeros(self.ms)
        if lib().orc_step(self.h, int(n), _dp(norm)):
            raise RuntimeError("Newton-Raphson projection did not converge")
        return norm

    def set_mag(self, mag):
        lib().orc_set_mag(self.h, float(mag))

    def sig(self):
        s = np.zeros(2); lib().orc_get_sig(self.h, _dp(s)); return s

    def maxdiff(self, other):
        flat = np.ascontiguousarray(np.asarray(other, np.complex128).reshape(-1, order="F"))
        return lib().orc_maxdiff(self.h, _dp(flat.view(np.float64)))


def fft1d(x, sign=-1):
    a = np.ascontiguousarray(np.asarray(x, np.complex128).copy())
    lib().orc_fft1d(a.size, _dp(a.view(np.float64)), sign)
    return a


def simpson(f, dx):
    f = np.ascontiguousarray(f, np.float64)
    return lib().orc_simpson(_dp(f), f.size, dx)


def diff(p, dx):
    p = np.ascontiguousarray(p, np.float64)
    d = np.empty_like(p)
    lib().orc_diff(_dp(p), p.size, dx, _dp(d))
    return d


def expm_se2(c6, cdt, v):
    c = np.ascontiguousarray(np.asarray(c6, np.complex128))
    out = np.ascontiguousarray(np.asarray(v, np.complex128).copy())
    lib().orc_expm_se2(_dp(c.view(np.float64)), complex(cdt).real, complex(cdt).imag, _dp(out.view(np.float64)))
    return out


def set_threads(n):
    lib().orc_set_num_threads(int(n))


def num_threads():
    return lib().orc_num_threads()


# ---------------------------------------------------------- the main loop
def run_loop(orc: Oracle, niter, stp, tol, dt, imag, record_every_step=False):
    """Restatement of the time loop (cgpe1d.f90:428-531) for the SO-coupled
    branch.  Returns dict with rows of file2 (t, EN/2, RMS...), file3 (t,
    NORM..., sum, MZ), convergence (t, CONV, CONV_EN), the final II-1 and
    final observables."""
    ms = orc.ms
    if imag:
        orc.normt()                       # cgpe1d.f90:394
    norm = orc.normc()
    rms = orc.rad()
    en, mu, mz = orc.energy()
    out = dict(initial=dict(norm=norm.copy(), en=en, mu=mu.copy(), mz=mz, rms=rms.copy()),
               file2=[], file3=[], conv=[])
    out["file2"].append([0.0, en / 2.0] + list(rms))
    out["file3"].append([0.0] + list(norm) + [norm.sum(), mz])
    en_old = 0.0
    phi_old = np.zeros(orc.shape + (ms,), np.complex128) if imag else None
    ii = 0
    exited = False
    for ii in range(1, niter + 1):
        if imag and stp > 0 and ii % stp == 0:
            phi_old = orc.state()             # one-step-old copy (cgpe1d.f90:508)
        norm = orc.step(1)
        if ii % stp == 0:
            en, mu, mz = orc.energy()
            rms = orc.rad()
            if imag:
                conv = orc.maxdiff(phi_old) / (stp * 2.0 * dt)
                conv_en = abs(en - en_old) / (stp * 2.0 * dt)
                out["conv"].append([2.0 * ii * dt, conv, conv_en])
                if conv <= tol or conv_en <= tol:
                    exited = True
                    break
            out["file2"].append([2.0 * ii * dt, en / 2.0] + list(rms))
            out["file3"].append([2.0 * ii * dt] + list(norm) + [norm.sum(), mz])
        en_old = en
    if not exited:
        ii = niter + 1
    en, mu, mz = orc.energy()
    rms = orc.rad()
    out["final"] = dict(ii_minus_1=ii - 1, norm=norm.copy(), en=en, mu=mu.copy(), mz=mz, rms=rms.copy())
    return out

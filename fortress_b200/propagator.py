"""Host-side mirror of the reference's propagator interface.

The FORTRESS programs drive the state through argument-less subroutines over
module globals (interfaces at SRC/cgpe1d.f90:117-198): FFT, KE, SOC, BFT, SE,
SP, NORMC, NORMT, RAD, ENERGY.  :class:`Propagator` owns one device-resident
instance through the C ABI (include/fgpe.h) and offers the same operations:

* ``step(n)``        n whole split steps FFT->KE->SOC->BFT->SE->SP->NORMC
                     [->NORMT], fused on the GPU (cgpe1d.f90:433-474)
* ``normc()``        NORMC of the last step before renormalisation
* ``normt()``        NORMT, returns TNORM
* ``energy()``       ENERGY -> (EN, MU, MZ)   (values as the reference returns
                     them; the files print EN/2 and MU/2)
* ``rad()``          RAD -> RMS
* ``conv()``         max |PHI - PHI_OLD| of the last step
* ``FFT() KE() SOC() BFT() SE() SP()``  the unfused single operators

Errors raise :class:`FgpeError`; nothing falls back to the CPU.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import FgpeError, check


def _dp(a):
    return a.ctypes.data_as(ctypes.POINTER(ctypes.c_double))


def make_params(dim, spin, n, d, dt, imag_time, tau, gamma=(0.0, 0.0, 0.0),
                alpha=(1.0, 1.0, 1.0), precision="fp64", kernels="auto", mag=0.0):
    """Fill an fgpe_params structure (include/fgpe.h)."""
    p = _abi.Params()
    n = list(n) + [1] * (3 - len(n))
    d = list(d) + [1.0] * (3 - len(d))
    g = list(gamma) + [0.0] * (3 - len(gamma))
    t = list(tau) + [0.0] * (3 - len(tau))
    p.dim, p.spin = int(dim), int(spin)
    p.nx, p.ny, p.nz = (int(v) for v in n)
    p.dx, p.dy, p.dz = (float(v) for v in d)
    p.dt = float(dt)
    p.imag_time = int(bool(imag_time))
    for i in range(3):
        p.tau[i] = float(t[i])
        p.gamma[i] = float(g[i])
        p.alpha[i] = float(alpha[i])
    p.precision = _abi.FGPE_FP32 if str(precision).lower() in ("fp32", "float32", "1") else _abi.FGPE_FP64
    p.kernels = {"auto": 0, "generic": 1, "fast-row": 2, "fast-col": 3, "split-1d": 4, "single-1d": 5, "cluster-1d": 6,
                 "warp-row": 7, "block-row": 8}[kernels]
    p.mag = float(mag)
    return p


class Propagator:
    def __init__(self, dim, spin, n, d, dt, imag_time, tau, gamma=(0.0, 0.0, 0.0),
                 alpha=(1.0, 1.0, 1.0), precision="fp64", kernels="auto", mag=0.0, _handle=None, _owner=None):
        L = _abi.load()
        p = make_params(dim, spin, n, d, dt, imag_time, tau, gamma, alpha, precision, kernels, mag)
        self.params = p
        self.dim, self.spin, self.ms = p.dim, p.spin, 2 * p.spin + 1
        self.shape = (p.nx, p.ny if p.dim >= 2 else 1, p.nz if p.dim >= 3 else 1)
        self._L = L
        self._owner = _owner
        if _handle is not None:          # an instance owned by a Batch
            self._h = _handle
            return
        h = ctypes.c_void_p()
        check(L.fgpe_create(ctypes.byref(p), ctypes.byref(h)))
        self._h = h

    @classmethod
    def from_config(cls, cfg, precision="fp64"):
        return cls(**cfg.params(precision))

    def close(self):
        if getattr(self, "_h", None):
            if self._owner is None:
                self._L.fgpe_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ck(self, rc):
        return check(rc, self._h)

    @property
    def handle(self):
        return self._h

    @property
    def npts(self):
        return int(np.prod(self.shape))

    # ------------------------------------------------------------- state
    def set_state(self, phi):
        a = np.asarray(phi, np.complex128).reshape(self.shape + (self.ms,), order="F")
        flat = np.ascontiguousarray(a.reshape(-1, order="F"))
        self._ck(self._L.fgpe_set_state(self._h, flat.ctypes.data))

    def set_state_host_ptr(self, ptr):
        """Upload from a raw host pointer (complex128, PHI layout)."""
        self._ck(self._L.fgpe_set_state(self._h, ctypes.c_void_p(ptr)))

    def state(self):
        flat = np.empty(self.npts * self.ms, np.complex128)
        self._ck(self._L.fgpe_get_state(self._h, flat.ctypes.data))
        return flat.reshape(self.shape + (self.ms,), order="F")

    def get_state_host_ptr(self, ptr):
        self._ck(self._L.fgpe_get_state(self._h, ctypes.c_void_p(ptr)))

    def set_state_device(self, ptr):
        self._ck(self._L.fgpe_set_state_device(self._h, ctypes.c_void_p(ptr)))

    def get_state_device(self, ptr):
        self._ck(self._L.fgpe_get_state_device(self._h, ctypes.c_void_p(ptr)))

    def set_stream(self, stream_ptr):
        self._ck(self._L.fgpe_set_stream(self._h, ctypes.c_void_p(stream_ptr)))

    # --------------------------------------------------------- operators
    def step(self, n=1, snapshot=True):
        flags = _abi.FGPE_STEP_DEFAULT if snapshot else _abi.FGPE_STEP_NO_SNAPSHOT
        self._ck(self._L.fgpe_step_ex(self._h, int(n), flags))

    def normt(self):
        t = np.zeros(1)
        self._ck(self._L.fgpe_normalize(self._h, _dp(t)))
        return float(t[0])

    def normc(self):
        n = np.zeros(self.ms)
        self._ck(self._L.fgpe_norms(self._h, _dp(n)))
        return n

    def observables(self):
        en = np.zeros(1); mz = np.zeros(1); mu = np.zeros(self.ms); rms = np.zeros(self.ms)
        self._ck(self._L.fgpe_observables(self._h, _dp(en), _dp(mu), _dp(mz), _dp(rms)))
        return float(en[0]), mu, float(mz[0]), rms

    def energy(self):
        en, mu, mz, _ = self.observables()
        return en, mu, mz

    def rad(self):
        return self.observables()[3]

    def conv(self):
        c = np.zeros(1)
        self._ck(self._L.fgpe_conv(self._h, _dp(c)))
        return float(c[0])

    def center(self):
        out = np.zeros(2 * self.ms)
        self._ck(self._L.fgpe_center(self._h, _dp(out)))
        return out[0::2] + 1j * out[1::2]

    def apply_op(self, name):
        self._ck(self._L.fgpe_apply_op(self._h, _abi.OPS[name]))

    def FFT(self): self.apply_op("FFT")
    def KE(self): self.apply_op("KE")
    def SOC(self): self.apply_op("SOC")
    def BFT(self): self.apply_op("BFT")
    def SE(self): self.apply_op("SE")
    def SP(self): self.apply_op("SP")

    def norms_async(self, ptr):
        """Enqueue the last step's NORMC into pinned/device memory at ptr."""
        self._ck(self._L.fgpe_norms_async(self._h, ctypes.c_void_p(ptr)))

    def norms_sink(self, ptr, count):
        """From now on every step appends its NORMC to the ring of count
        records at ptr (pinned host or device memory); ptr = 0 stops it."""
        self._ck(self._L.fgpe_norms_sink(self._h, ctypes.c_void_p(ptr or None), int(count)))

    def profile(self, on=True):
        self._ck(self._L.fgpe_profile_enable(self._h, int(on)))

    def profile_read(self, reset=True):
        """Per kernel class (row, col-y, col-z, 1D): (total ms, launches)."""
        ms = np.zeros(4)
        n = (ctypes.c_longlong * 4)()
        self._ck(self._L.fgpe_profile_read(self._h, _dp(ms), n, int(reset)))
        return ms, np.array(list(n))

    def set_kernels(self, kernels):
        self._ck(self._L.fgpe_set_kernels(self._h, {"auto": 0, "generic": 1, "fast-row": 2, "fast-col": 3,
                                                    "warp-row": 7, "block-row": 8}[kernels]))

    def save(self, path, step=0, user=None):
        """Full-precision checkpoint (fgpe_checkpoint_save); user: up to 8 floats."""
        u = np.zeros(8)
        if user is not None:
            u[:len(user)] = user
        self._ck(self._L.fgpe_checkpoint_save(self._h, str(path).encode(), int(step), _dp(u)))

    def load(self, path):
        """Restore a checkpoint; returns (step, user[8])."""
        st = ctypes.c_longlong()
        u = np.zeros(8)
        self._ck(self._L.fgpe_checkpoint_load(self._h, str(path).encode(), ctypes.byref(st), _dp(u)))
        return int(st.value), u

    def kernel_launches(self):
        c = ctypes.c_longlong()
        self._ck(self._L.fgpe_kernel_launches(self._h, ctypes.byref(c)))
        return int(c.value)


def device_ok():
    try:
        return bool(_abi.load().fgpe_device_ok())
    except FgpeError:
        return False

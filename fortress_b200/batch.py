"""Batched sweeps: many independent instances advanced by one CUDA-graph
launch per group of steps (C ABI: fgpe_batch_* in include/fgpe.h).

The reference runs one parameter point per process; a phase-diagram sweep
over spin-orbit strengths, couplings and trap anisotropies with uneven grid
sizes is a batch here.  Each instance is a full :class:`Propagator`.
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _abi
from ._abi import check_batch
from .propagator import Propagator, make_params


class Batch:
    def __init__(self, instances):
        """instances: list of keyword dicts for :class:`Propagator`."""
        L = _abi.load()
        arr = (_abi.Params * len(instances))()
        for i, kw in enumerate(instances):
            arr[i] = make_params(**kw)
        b = ctypes.c_void_p()
        check_batch(L.fgpe_batch_create(arr, len(instances), ctypes.byref(b)))
        self._b, self._L = b, L
        self.props = []
        for i, kw in enumerate(instances):
            h = ctypes.c_void_p()
            check_batch(L.fgpe_batch_instance(b, i, ctypes.byref(h)), b)
            self.props.append(Propagator(**kw, _handle=h, _owner=self))

    def __len__(self):
        return len(self.props)

    def __getitem__(self, i):
        return self.props[i]

    def close(self):
        if getattr(self, "_b", None):
            for p in self.props:
                p._h = None
            self._L.fgpe_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def config(self, width=0, steps_per_graph=0):
        check_batch(self._L.fgpe_batch_config(self._b, int(width), int(steps_per_graph)), self._b)

    def mode(self, grouped=False, persistent=False):
        """grouped=True: instances sharing a q2D grid shape advance together,
        one column-pass and one row-pass launch per step per group;
        persistent=True: every q2D instance of a size-specialised grid (one
        spin and precision) advances by one persistent kernel launch per
        graph of steps; neither: one graph branch per instance
        (fgpe_batch_mode)."""
        if persistent:
            m = _abi.FGPE_BATCH_PERSISTENT
        else:
            m = _abi.FGPE_BATCH_GROUPED if grouped else _abi.FGPE_BATCH_BRANCHES
        check_batch(self._L.fgpe_batch_mode(self._b, m), self._b)

    def variant(self, v=-1):
        """Select the persistent kernel variant v (v < 0: keep it); returns
        the current one (fgpe_batch_variant)."""
        cur = ctypes.c_int()
        check_batch(self._L.fgpe_batch_variant(self._b, int(v), ctypes.byref(cur)), self._b)
        return cur.value

    @staticmethod
    def variant_shapes():
        """Shapes of the persistent kernel variants: dicts of threads per
        block, values per row tile, bytes of x per column tile row and the
        radix plan of the y lines (fgpe_batch_variant_shape)."""
        L = _abi.load()
        out = []
        for v in range(L.fgpe_batch_variants()):
            sh = (ctypes.c_int * 4)()
            check_batch(L.fgpe_batch_variant_shape(v, sh))
            out.append(dict(threads=sh[0], row_values=sh[1], col_bytes=sh[2], y_plan=sh[3]))
        return out

    def wait_bound(self, wait_ms, stall_instance=-1):
        """Bound on one device-side wait of the persistent kernel, in ms;
        stall_instance >= 0 makes that instance's first wait run out (a test
        of the error path: the next step raises FgpeError FGPE_E_TIMEOUT)."""
        check_batch(self._L.fgpe_batch_wait_bound(self._b, float(wait_ms), int(stall_instance)), self._b)

    def tuning(self):
        w, k = ctypes.c_int(), ctypes.c_int()
        check_batch(self._L.fgpe_batch_tuning(self._b, ctypes.byref(w), ctypes.byref(k)), self._b)
        return w.value, k.value

    def autotune(self, trial_steps=8, cache_path=None):
        c = cache_path.encode() if cache_path else None
        check_batch(self._L.fgpe_batch_autotune(self._b, int(trial_steps), c), self._b)
        return self.tuning()

    def step(self, n):
        check_batch(self._L.fgpe_batch_step(self._b, int(n)), self._b)

    def step_timed(self, n):
        """n steps as whole graph launches; returns their device time in ms."""
        ms = ctypes.c_double()
        check_batch(self._L.fgpe_batch_step_timed(self._b, int(n), ctypes.byref(ms)), self._b)
        return ms.value

    def observables(self, with_conv=True):
        """Per instance: dict(en, mz, conv, mu, rms, norm)."""
        ms = [p.ms for p in self.props]
        stride = [3 + 3 * m for m in ms]
        out = np.zeros(sum(stride))
        check_batch(self._L.fgpe_batch_observables(self._b, out.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
                                                   int(bool(with_conv))), self._b)
        res, o = [], 0
        for m, s in zip(ms, stride):
            v = out[o:o + s]
            res.append(dict(en=v[0], mz=v[1], conv=v[2], mu=v[3:3 + m].copy(), rms=v[3 + m:3 + 2 * m].copy(),
                            norm=v[3 + 2 * m:3 + 3 * m].copy()))
            o += s
        return res

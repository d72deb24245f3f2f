"""The reference's time loop on top of :class:`Propagator`.

Restates PROGRAM CGPE1D/2D/3D's loop for the spin-orbit-coupled branch
(cgpe1d.f90:394-531; 2D 401-545; 3D 412-581): initial NORMT in imaginary
time, NORMC/RAD/ENERGY of the initial state, then per step the fused split
step; every STP steps ENERGY, RAD and, in imaginary time, CONV =
max|PHI-PHI_OLD|/(STP*2*DT) and CONV_EN = |EN-EN_OLD|/(STP*2*DT) with exit on
either <= TOL before the file2/file3 rows are written.  The device keeps the
state; the host only reads scalars at STP boundaries (the reference's
one-step-old PHI_OLD copy every step is replaced by a snapshot at the step
before each STP boundary).
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np


@dataclass
class RunResult:
    initial: dict = field(default_factory=dict)
    file2: list = field(default_factory=list)     # t, EN/2, RMS...
    file3: list = field(default_factory=list)     # t, NORM..., sum, MZ
    conv: list = field(default_factory=list)      # t, CONV, CONV_EN
    nstp_rows: list = field(default_factory=list) # every NSTP: (ii, norm, en, mu, |phi(center)|)
    final: dict = field(default_factory=dict)


def run(prop, niter, stp, tol, dt, imag, nstp=0, on_nstp=None):
    res = RunResult()
    if imag:
        prop.normt()
    norm = prop.normc()
    en, mu, mz, rms = prop.observables()
    res.initial = dict(norm=norm, en=en, mu=mu, mz=mz, rms=rms, center=np.abs(prop.center()))
    res.file2.append([0.0, en / 2.0] + list(rms))
    res.file3.append([0.0] + list(norm) + [norm.sum(), mz])
    en_old = en
    ii = 0
    exited = False
    while ii < niter:
        # advance to the next STP or NSTP boundary in one fused batch
        nxt = min(niter, (ii // stp + 1) * stp)
        if nstp:
            nxt = min(nxt, (ii // nstp + 1) * nstp)
        prop.step(nxt - ii)
        ii = nxt
        norm = None
        if ii % stp == 0:
            norm = prop.normc()
            en, mu, mz, rms = prop.observables()
            if imag:
                c = prop.conv() / (stp * 2.0 * dt)
                # EN_OLD starts at 0 and takes EN after every step
                # (cgpe1d.f90:294, 507): only a boundary at II = 1 sees the 0
                ce = abs(en - (en_old if ii > 1 else 0.0)) / (stp * 2.0 * dt)
                res.conv.append([2.0 * ii * dt, c, ce])
                if c <= tol or ce <= tol:
                    exited = True
                    break
            res.file2.append([2.0 * ii * dt, en / 2.0] + list(rms))
            res.file3.append([2.0 * ii * dt] + list(norm) + [norm.sum(), mz])
            en_old = en
        if nstp and ii % nstp == 0:
            if norm is None:
                norm = prop.normc()
            row = (ii, norm.copy(), en, mu.copy(), np.abs(prop.center()))
            res.nstp_rows.append(row)
            if on_nstp:
                on_nstp(ii, prop)
    ii_minus_1 = ii - 1 if exited else niter
    en, mu, mz, rms = prop.observables()
    res.final = dict(ii_minus_1=ii_minus_1, norm=prop.normc(), en=en, mu=mu, mz=mz, rms=rms,
                     center=np.abs(prop.center()), exited=exited)
    return res

"""FP32-bulk path against the FP64 path: errors of every reported quantity.

The FP32 path keeps FFTs and the pointwise exponentials in complex64 and the
NORMC/ENERGY/RAD/MZ reductions, the imaginary-time renormalisation and the
convergence test in FP64.  The FP64 path is the reference here (it matches the
CPU restatement of the reference to 1e-11, see the parity tests).  Prints one
JSON object per case.

    python -m fortress_b200.experiments.precision [--steps N]
"""
from __future__ import annotations

import argparse
import json

import numpy as np

import fortress_b200 as F
from fortress_b200.config import RunConfig


def _guess(p, seed=3):
    rng = np.random.default_rng(seed)
    axes = [(np.arange(n) - n / 2) * d for n, d in zip(p["n"], p["d"])]
    r2 = 0
    for a, x in enumerate(axes):
        shape = [1] * len(axes)
        shape[a] = -1
        r2 = r2 + p["alpha"][a] * (x.reshape(shape) ** 2)
    g = np.exp(-r2 / 2.0)
    ms = 2 * p["spin"] + 1
    phi = np.stack([g * (1 + 1e-3 * rng.uniform(size=g.shape)) for _ in range(ms)], axis=-1).astype(complex)
    return phi.reshape(tuple(p["n"]) + (1,) * (3 - len(p["n"])) + (ms,))


def cases():
    q2d = RunConfig(dim=2, spin=2, n=(512, 512, 1), d=(0.05, 0.05, 1.0), dt=1e-4, mass=87.0,
                    a=(87.93, 91.28, 99.18), natoms=50000, nu=(20.0, 20.0, 500.0), switch_im=0,
                    gamma=(1.2, 1.0, 0.0))
    d3 = RunConfig(dim=3, spin=1, n=(128, 128, 128), d=(0.2, 0.2, 0.2), dt=1e-3, mass=87.0,
                   a=(101.8, 100.4, 0.0), natoms=100000, nu=(50.0, 50.0, 50.0), switch_im=1,
                   gamma=(0.5, 0.5, 0.5))
    return [("q2d-spin2-realtime-512x512", q2d), ("3d-spin1-imag-128^3", d3)]


def compare(name, cfg, steps):
    p64 = cfg.params("fp64")
    p32 = cfg.params("fp32")
    phi = _guess(p64)
    a, b = F.Propagator(**p64), F.Propagator(**p32)
    a.set_state(phi); b.set_state(phi)
    # start both from the unit-norm state: a real-time run of the reference
    # continues a normalised imaginary-time solution
    a.normt(); b.normt()
    a.step(steps); b.step(steps)
    ea, mua, mza, ra = a.observables()
    eb, mub, mzb, rb = b.observables()
    na, nb = a.normc(), b.normc()
    sa, sb = a.state(), b.state()
    rel = lambda x, y: float(np.max(np.abs(np.asarray(x) - np.asarray(y)) / np.maximum(np.abs(np.asarray(y)), 1e-300)))
    return dict(case=name, steps=steps, energy_rel=rel(eb, ea), mu_rel=rel(mub, mua), rms_rel=rel(rb, ra),
                norm_rel=rel(nb, na), mz_abs=abs(mzb - mza),
                density_maxabs=float(np.max(np.abs(np.abs(sb) ** 2 - np.abs(sa) ** 2))),
                density_peak=float(np.max(np.abs(sa) ** 2)))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--steps", type=int, default=1000)
    args = ap.parse_args()
    for name, cfg in cases():
        print(json.dumps(compare(name, cfg, args.steps)))


if __name__ == "__main__":
    main()

"""FP32-bulk path (complex64 FFTs and exponentials; FP64 NORMC, ENERGY, RAD,
MZ, renormalisation and CONV) against the FP64 oracle: the error of every
reported quantity, printed as one JSON line per case and held to the bounds
written beside each case.

* q2D spin-2 SO-coupled real-time quench on the benchmark's 512^2 grid
  (DT=1e-4, Rb-87, GAMMAX 1.2, GAMMAY 1.0), 200 steps from the unit-norm
  Gaussian start.
* 3D spin-1 SO-coupled imaginary time with the 256^3 workload's physics on a
  64^3 grid of the same box (DX=0.4, DT=1e-3), 1000 steps from the seeded
  Gaussian.
"""
import json

import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import oracle_kwargs

pytestmark = pytest.mark.gpu


def _rel(a, b):
    a, b = np.asarray(a, float), np.asarray(b, float)
    return float(np.max(np.abs(a - b) / np.maximum(np.abs(b), 1e-300)))


def _cases():
    from fortress_b200.config import RunConfig
    q2d = RunConfig(dim=2, spin=2, n=(512, 512, 1), d=(0.05, 0.05, 1.0), dt=1e-4, mass=87.0,
                    a=(87.93, 91.28, 99.18), natoms=50000, nu=(20.0, 20.0, 500.0), switch_im=0,
                    gamma=(1.2, 1.0, 0.0))
    d3 = RunConfig(dim=3, spin=1, n=(64, 64, 64), d=(0.4, 0.4, 0.4), dt=1e-3, mass=87.0, a=(101.8, 100.4, 0.0),
                   natoms=100000, nu=(50.0, 50.0, 50.0), switch_im=1, gamma=(0.5, 0.5, 0.5))
    # (name, config, steps, bounds: energy, mu, rms, norm, density / peak)
    # bounds about 2.5x the measured errors: q2D energy 2.0e-5, mu 2.3e-5, rms
    # 1.4e-5, norm 2.8e-5, density 4.2e-5; 3D energy 6.9e-8, mu 3.0e-7, rms
    # 1.8e-5, norm 3.6e-5, density 4.4e-5
    return [("q2d-spin2-realtime-512^2", q2d, 200, (5e-5, 6e-5, 4e-5, 7e-5, 1e-4)),
            ("3d-spin1-imag-64^3", d3, 1000, (2e-7, 1e-6, 5e-5, 1e-4, 1e-4))]


def _start(p, seed=3):
    axes = [(-1.0 + 2.0 * np.arange(n) / n) * n * d / 2.0 for n, d in zip(p["n"], p["d"])]
    r2 = 0
    for a, x in enumerate(axes):
        shape = [1] * len(axes)
        shape[a] = -1
        r2 = r2 + x.reshape(shape) ** 2
    g = np.exp(-r2 / 2.0)
    rng = np.random.default_rng(seed)
    ms = 2 * p["spin"] + 1
    phi = np.stack([g * (1.0 + 1e-3 * rng.uniform(size=g.shape)) for _ in range(ms)], axis=-1).astype(complex)
    return phi.reshape(tuple(p["n"]) + (1,) * (3 - len(p["n"])) + (ms,))


@pytest.mark.parametrize("case", _cases(), ids=lambda c: c[0])
def test_fp32_bulk_errors_against_oracle(case):
    import fortress_b200 as F
    name, cfg, steps, bounds = case
    p64 = cfg.params("fp64")
    phi = _start(p64)
    orc = O.Oracle(**oracle_kwargs(p64))
    orc.set_state(phi)
    orc.normt()                          # a unit-norm start for both
    phi = orc.state()
    prop = F.Propagator(**cfg.params("fp32"))
    try:
        prop.set_state(phi)
        prop.step(steps)
        en, mu, mz, rms = prop.observables()
        norm = prop.normc()
        dens = np.abs(prop.state()) ** 2
    finally:
        prop.close()
    norm_o = orc.step(steps)
    en_o, mu_o, mz_o = orc.energy()
    rms_o = orc.rad()
    dens_o = np.abs(orc.state()) ** 2
    err = {"case": name, "steps": steps, "energy_rel": _rel(en, en_o), "mu_rel": _rel(mu, mu_o),
           "rms_rel": _rel(rms, rms_o), "norm_rel": _rel(norm, norm_o), "mz_abs": abs(mz - mz_o),
           "density_maxabs_over_peak": float(np.abs(dens - dens_o).max() / dens_o.max())}
    print(json.dumps({"fp32_vs_oracle": err}))
    b = bounds
    assert err["energy_rel"] <= b[0] and err["mu_rel"] <= b[1] and err["rms_rel"] <= b[2]
    assert err["norm_rel"] <= b[3] and err["density_maxabs_over_peak"] <= b[4]

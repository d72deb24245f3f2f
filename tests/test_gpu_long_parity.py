"""Long runs of the q2D spin-2 real-time workload against the CPU oracle.

The workload's own start: the imaginary-time ground state at gamma = (1, 1)
plus seeded 1e-3 complex noise, then a quench of GAMMAX to 1.2.
* At the full 512^2 size, 500 steps.
* On a 128^2 grid of the same box, 10 000 steps.
From this start the GPU/oracle difference grows linearly. Measured: 9.7e-14
relative energy at 1000 steps on 512^2; 3.4e-12 at 10 000 steps and 7.6e-12
at 20 000 steps on 128^2.

A third case quenches the plain Gaussian guess for 50 steps at 512^2.  That
state is far from equilibrium and amplifies any rounding difference by about
x10 per 100 steps after step ~400.  Two FP64 implementations that differ only
in summation order then separate, so it is only a short-run case.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import oracle_kwargs

pytestmark = pytest.mark.gpu


def _params(n, gamma=(1.2, 1.0)):
    from fortress_b200.config import RunConfig
    c = RunConfig(dim=2, spin=2, n=(n, n, 1), d=(25.6 / n, 25.6 / n, 1.0), dt=1e-4, mass=87.0,
                  a=(87.93, 91.28, 99.18), natoms=50000, nu=(20.0, 20.0, 500.0), switch_im=0,
                  gamma=(gamma[0], gamma[1], 0.0))
    return c.params("fp64")


def _gaussian(p, seed):
    n, d = p["n"][0], p["d"][0]
    x = (-1.0 + 2.0 * np.arange(n) / n) * n * d / 2.0
    g = np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / 2.0)
    rng = np.random.default_rng(seed)
    phi = np.stack([g * (1 + 1e-3 * (rng.standard_normal(g.shape) + 1j * rng.standard_normal(g.shape)))
                    for _ in range(5)], axis=-1)
    # plain l2 normalisation is enough for a start state
    return (phi / np.sqrt(np.sum(np.abs(phi) ** 2) * d * d)).reshape(n, n, 1, 5)


def _quench_start(F, n, seed=2):
    """Ground state at gamma = (1, 1): 3000 imaginary-time steps of dt = 1e-3
    from the default spin-2 guess, plus 1e-3 of the peak amplitude in seeded
    complex Gaussian noise."""
    p = dict(_params(n, (1.0, 1.0)), imag_time=True, dt=1e-3)
    d = p["d"][0]
    x = (-1.0 + 2.0 * np.arange(n) / n) * n * d / 2.0
    ax, ay = p["alpha"][0], p["alpha"][1]
    g = np.sqrt(0.2) * np.exp(-(ax * x[:, None] ** 2 + ay * x[None, :] ** 2) / 2.0) / np.sqrt(np.pi)
    r = F.Propagator(**p)
    try:
        r.set_state(np.repeat(g[:, :, None, None], 5, axis=3).astype(complex))
        r.normt()
        r.step(3000)
        phi = r.state()
    finally:
        r.close()
    rng = np.random.default_rng(seed)
    return phi + 1e-3 * np.abs(phi).max() * (rng.standard_normal(phi.shape) + 1j * rng.standard_normal(phi.shape))


def _compare(F, p, phi, steps, tol_e, tol_d):
    orc = O.Oracle(**oracle_kwargs(p))
    orc.set_state(phi)
    prop = F.Propagator(**p)
    try:
        prop.set_state(phi)
        orc.step(steps)
        prop.step(steps)
        en_g, mu_g, mz_g, rms_g = prop.observables()
        dens_g = np.abs(prop.state()) ** 2
    finally:
        prop.close()
    en_o, mu_o, mz_o = orc.energy()
    assert abs(en_g - en_o) <= tol_e * abs(en_o)
    assert np.allclose(mu_g, mu_o, rtol=10 * tol_e, atol=0)
    assert np.allclose(rms_g, orc.rad(), rtol=10 * tol_e, atol=0)
    dens_o = np.abs(orc.state()) ** 2
    assert np.abs(dens_g - dens_o).max() <= tol_d


def test_quench_full_size_matches_oracle():
    import fortress_b200 as F
    # measured: 4.6e-14 relative energy, 3.3e-15 max-abs density after 500 steps
    _compare(F, _params(512), _quench_start(F, 512), 500, tol_e=1e-11, tol_d=1e-12)


def test_quench_long_run_matches_oracle():
    import fortress_b200 as F
    # measured: 3.4e-12 relative energy, 4.9e-14 max-abs density after 10 000 steps
    _compare(F, _params(128), _quench_start(F, 128), 10000, tol_e=1e-10, tol_d=1e-12)


def test_gaussian_quench_short_run_matches_oracle():
    import fortress_b200 as F
    p = _params(512)
    # measured: 4e-14 relative energy, 5e-15 max-abs density after 50 steps
    _compare(F, p, _gaussian(p, 2), 50, tol_e=1e-11, tol_d=1e-12)

"""Replica scheduler on one GPU: the batched per-rank work gives the same
observables as stepping each instance alone."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _guess(p):
    n, d = p["n"][0], p["d"][0]
    x = (np.arange(n) - n / 2) * d
    g = np.exp(-(x[:, None] ** 2 + p["alpha"][1] * x[None, :] ** 2) / 2.0)
    return np.repeat(g[:, :, None], 3, axis=2).astype(complex)


def test_sweep_matches_individual_runs():
    import fortress_b200 as F
    from fortress_b200 import sweep
    insts = [dict(dim=2, spin=1, n=(n, n), d=(0.2, 0.2), dt=1e-3, imag_time=True, tau=(400.0, -8.0, 0.0),
                  gamma=(g, 0.5), alpha=(1.0, 1.3, 1.0)) for n, g in ((64, 0.3), (48, 0.8), (64, 1.2))]
    recs = sweep.run(insts, sweep.imaginary_time_work(40, _guess))
    for p, r in zip(insts, recs):
        a = F.Propagator(**p)
        a.set_state(_guess(p))
        a.normt()
        a.step(40)
        en, mu, mz, rms = a.observables()
        assert abs(r["en"] - en) <= 1e-12 * abs(en)
        np.testing.assert_allclose(r["mu"], mu, rtol=1e-12)
        np.testing.assert_allclose(r["rms"], rms, rtol=1e-12)

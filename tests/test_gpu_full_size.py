"""The 3D spin-1 imaginary-time workload at its full 256^3 size.

At 256^3 the step runs kernels that no smaller 3D case reaches: the
size-specialised row kernel on 256-point x lines and the 128-byte-wide column
tiles on 256-point y and z lines.  The GPU path is held to the oracle for a
few steps at that size (states 1e-11 relative, observables 1e-10), and the
FP32 bulk path to the FP64 path with the FP32 tolerances.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import oracle_kwargs, rel_err

pytestmark = pytest.mark.gpu


def _params(precision="fp64"):
    from fortress_b200.config import RunConfig
    c = RunConfig(dim=3, spin=1, n=(256, 256, 256), d=(0.1, 0.1, 0.1), dt=1e-3, mass=87.0,
                  a=(101.8, 100.4, 0.0), natoms=100000, nu=(50.0, 50.0, 50.0), switch_im=1,
                  gamma=(0.5, 0.5, 0.5))
    return c.params(precision)


def _state(p, seed):
    """Gaussian of width 1 per component with seeded amplitude noise and
    phases, so that every operator sees a generic complex spinor."""
    n, d = p["n"][0], p["d"][0]
    x = (np.arange(n) - n // 2) * d
    g = np.exp(-(x[:, None, None] ** 2 + x[None, :, None] ** 2 + x[None, None, :] ** 2) / 2.0)
    rng = np.random.default_rng(seed)
    phi = np.empty(g.shape + (3,), dtype=complex)
    for m in range(3):
        phi[..., m] = g * (1.0 + 0.05 * rng.standard_normal(g.shape)) * np.exp(1j * rng.uniform(-0.4, 0.4, g.shape))
    return phi


def test_full_size_3d_matches_oracle():
    import fortress_b200 as F
    p = _params()
    phi = _state(p, 7)
    orc = O.Oracle(**oracle_kwargs(p))
    orc.set_state(phi)
    prop = F.Propagator(**p)
    try:
        prop.set_state(phi)
        orc.normt()
        prop.normt()
        norm_o = orc.step(3)
        prop.step(3)
        assert rel_err(prop.state(), orc.state()) < 1e-11
        assert np.allclose(prop.normc(), norm_o, rtol=1e-11, atol=0)
        en_g, mu_g, mz_g, rms_g = prop.observables()
    finally:
        prop.close()
    en_o, mu_o, mz_o = orc.energy()
    assert abs(en_g - en_o) <= 1e-10 * abs(en_o)
    assert np.allclose(mu_g, mu_o, rtol=1e-10, atol=1e-12)
    assert abs(mz_g - mz_o) <= 1e-10 * max(1.0, abs(mz_o))
    assert np.allclose(rms_g, orc.rad(), rtol=1e-10, atol=0)


def test_full_size_3d_fp32_bulk_against_fp64():
    import fortress_b200 as F
    phi = _state(_params(), 8)
    out = {}
    for precision in ("fp64", "fp32"):
        prop = F.Propagator(**_params(precision))
        try:
            prop.set_state(phi)
            prop.normt()
            prop.step(20)
            out[precision] = (prop.state(), prop.observables())
        finally:
            prop.close()
    (s64, o64), (s32, o32) = out["fp64"], out["fp32"]
    assert rel_err(s32, s64) < 2e-5
    assert abs(o32[0] - o64[0]) <= 2e-5 * abs(o64[0])
    assert np.allclose(o32[3], o64[3], rtol=2e-5)

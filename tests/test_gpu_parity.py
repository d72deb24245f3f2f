"""GPU path (libfgpe.so through the C ABI) against the CPU oracle on the same
seeded inputs.  FP64 tolerances: states 1e-11 relative to max|phi| per step
batch, observables 1e-10 relative; FP32 bulk path: 2e-5."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import CASES, case_id, case_params, initial_state, oracle_kwargs, rel_err

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    import fortress_b200 as F
    if not F.device_ok():
        pytest.fail("no usable sm_100 device / libfgpe.so not loaded")
    return F


def _pair(F, case, precision="fp64", seed=0):
    p = case_params(case)
    orc = O.Oracle(**oracle_kwargs(p))
    phi = initial_state(orc, seed)
    orc.set_state(phi)
    prop = F.Propagator(**p, precision=precision)
    prop.set_state(phi)
    return orc, prop


@pytest.mark.parametrize("case", CASES, ids=case_id)
@pytest.mark.parametrize("op", ["FFT", "KE", "SOC", "BFT", "SE", "SP"])
def test_operator(F, case, op):
    orc, prop = _pair(F, case)
    if op in ("KE", "SOC", "BFT"):
        orc.fft(); prop.FFT()
    getattr(orc, op.lower())()
    getattr(prop, op)()
    assert rel_err(prop.state(), orc.state()) < 1e-12


@pytest.mark.parametrize("case", CASES, ids=case_id)
def test_steps(F, case):
    orc, prop = _pair(F, case)
    dim, spin, imag, n = case
    if imag:
        orc.normt(); prop.normt()
    for batch in (1, 7):
        prev = orc.state()
        norm_o = orc.step(batch)
        prop.step(batch)
        assert rel_err(prop.state(), orc.state()) < 1e-11
        assert np.allclose(prop.normc(), norm_o, rtol=1e-11, atol=0)
        en_g, mu_g, mz_g, rms_g = prop.observables()
        en_o, mu_o, mz_o = orc.energy()
        assert abs(en_g - en_o) <= 1e-10 * abs(en_o)
        assert np.allclose(mu_g, mu_o, rtol=1e-10, atol=1e-12)
        assert abs(mz_g - mz_o) <= 1e-10 * max(1.0, abs(mz_o))
        assert np.allclose(rms_g, orc.rad(), rtol=1e-10, atol=0)
        if batch == 1:
            c_o = orc.maxdiff(prev)
            assert abs(prop.conv() - c_o) <= 1e-9 * c_o + 1e-15


@pytest.mark.parametrize("case", [CASES[i] for i in (1, 5, 6, 9)], ids=case_id)
def test_fp32_bulk(F, case):
    orc, prop = _pair(F, case, precision="fp32")
    dim, spin, imag, n = case
    if imag:
        orc.normt(); prop.normt()
    orc.step(10)
    prop.step(10)
    assert rel_err(prop.state(), orc.state()) < 2e-5
    en_g, mu_g, mz_g, rms_g = prop.observables()
    en_o, mu_o, mz_o = orc.energy()
    assert abs(en_g - en_o) <= 2e-5 * abs(en_o)
    assert np.allclose(rms_g, orc.rad(), rtol=2e-5)


def test_error_paths(F):
    with pytest.raises(F.FgpeError):
        F.Propagator(dim=2, spin=1, n=(32, 14), d=(0.1, 0.1), dt=1e-3, imag_time=1, tau=(1, 0, 0))  # 14 = 2*7 has a factor outside {2,3,5}
    with pytest.raises(F.FgpeError):
        F.Propagator(dim=2, spin=3, n=(32, 32), d=(0.1, 0.1), dt=1e-3, imag_time=1, tau=(1, 0, 0))
    p = F.Propagator(dim=2, spin=1, n=(32, 32), d=(0.1, 0.1), dt=1e-3, imag_time=1, tau=(1, 0, 0))
    with pytest.raises(F.FgpeError):
        p.step(1)      # no state set


from tests.helpers import FAST_CASES  # noqa: E402


@pytest.mark.parametrize("case", FAST_CASES, ids=case_id)
def test_fast_kernels(F, case):
    orc, prop = _pair(F, case, seed=3)
    dim, spin, imag, n = case
    if imag:
        orc.normt(); prop.normt()
    norm_o = orc.step(3)
    prop.step(3)
    assert rel_err(prop.state(), orc.state()) < 1e-11
    assert np.allclose(prop.normc(), norm_o, rtol=1e-11, atol=0)
    en_g = prop.observables()[0]
    en_o = orc.energy()[0]
    assert abs(en_g - en_o) <= 1e-10 * abs(en_o)


@pytest.mark.parametrize("case", [FAST_CASES[0], FAST_CASES[4]], ids=case_id)
def test_fast_kernels_fp32(F, case):
    orc, prop = _pair(F, case, precision="fp32", seed=4)
    dim, spin, imag, n = case
    if imag:
        orc.normt(); prop.normt()
    orc.step(3)
    prop.step(3)
    assert rel_err(prop.state(), orc.state()) < 2e-5


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
def test_fast_matches_generic_512(F, precision):
    """Size-specialised and generic kernels agree on the 512^2 spin-2
    real-time bench workload (GPU only, 20 steps)."""
    p = case_params((2, 2, 0, (512, 512)))
    rng = np.random.default_rng(5)
    x = (np.arange(512) - 256) * p["d"][0]
    g = np.exp(-(x[:, None] ** 2 + x[None, :] ** 2) / 8.0)
    phi = np.stack([g * np.exp(1j * rng.uniform(-0.3, 0.3, g.shape)) for _ in range(5)], axis=-1)
    a = F.Propagator(**p, precision=precision)
    b = F.Propagator(**p, precision=precision, kernels="generic")
    a.set_state(phi); b.set_state(phi)
    a.step(20); b.step(20)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rel_err(a.state(), b.state()) < tol


WIDE_CASES = [((3, 1, 1, (128, 128, 128)), "fp64"), ((3, 2, 0, (128, 128, 128)), "fp64"),
              ((3, 1, 0, (256, 128, 128)), "fp32")]


@pytest.mark.parametrize("case,precision", WIDE_CASES, ids=lambda v: case_id(v) if isinstance(v, tuple) else v)
def test_wide_column_tiles_match_generic(F, case, precision):
    """3D grids with enough column tiles take the wide (128-byte) column
    tiles; they agree with the generic kernels (GPU only, 6 steps)."""
    p = case_params(case)
    rng = np.random.default_rng(6)
    axes = np.meshgrid(*[(np.arange(n) - n / 2) * d for n, d in zip(case[3], p["d"])], indexing="ij")
    g = np.exp(-sum(a ** 2 for a in axes) / 8.0)
    ms = 2 * case[1] + 1
    phi = np.stack([g * np.exp(1j * rng.uniform(-0.3, 0.3, g.shape)) for _ in range(ms)], axis=-1)
    a = F.Propagator(**p, precision=precision)
    b = F.Propagator(**p, precision=precision, kernels="generic")
    a.set_state(phi); b.set_state(phi)
    if case[2]:
        a.normt(); b.normt()
    a.step(6); b.step(6)
    tol = 1e-12 if precision == "fp64" else 1e-5
    assert rel_err(a.state(), b.state()) < tol
    assert np.allclose(a.normc(), b.normc(), rtol=tol)


PROJ_CASES = [(1, 1, 1, (96,)), (1, 2, 1, (64,)), (2, 1, 1, (32, 24)), (2, 2, 1, (32, 32)),
              (3, 1, 1, (16, 16, 12)), (3, 2, 1, (16, 12, 16)), (2, 2, 1, (128, 192))]


@pytest.mark.parametrize("case", PROJ_CASES, ids=case_id)
def test_projection_branch(F, case):
    """Imaginary time without SOC: SIGMA projection to the imposed MAG
    (spin-1 closed form, spin-2 Newton) before NORMT, cgpe1d.f90:443-470."""
    p = case_params(case)
    p["gamma"] = (0.0,) * case[0]
    mag = 0.3 if case[1] == 2 else 0.2
    orc = O.Oracle(**oracle_kwargs(p))
    phi = initial_state(orc, 1)
    orc.set_state(phi)
    orc.set_mag(mag)
    prop = F.Propagator(**p, mag=mag)
    prop.set_state(phi)
    orc.normt(); prop.normt()
    for batch in (1, 6):
        norm_o = orc.step(batch)
        prop.step(batch)
        assert np.allclose(prop.normc(), norm_o, rtol=1e-11, atol=0)
        assert rel_err(prop.state(), orc.state()) < 1e-11
    en_g, mu_g, mz_g, _ = prop.observables()
    en_o, mu_o, mz_o = orc.energy()
    assert abs(mz_g - mag) < 1e-12 and abs(mz_o - mag) < 1e-12
    assert abs(en_g - en_o) <= 1e-10 * abs(en_o)


@pytest.mark.parametrize("case", [(2, 2, 1, (64, 48)), (3, 1, 0, (16, 16, 12)), (1, 2, 1, (4096,))], ids=case_id)
def test_bulk_graph_replay_is_bitwise_eager(F, case):
    """Multi-step calls replay a captured graph of whole steps for their bulk;
    with kernel profiling on the same steps run eagerly.  Same kernels, same
    order: bitwise the same state, norms and CONV."""
    p = case_params(case)
    orc = O.Oracle(**oracle_kwargs(p))
    phi = initial_state(orc, 4)
    a, b = F.Propagator(**p), F.Propagator(**p)
    a.set_state(phi); b.set_state(phi)
    b.profile(True)
    for n in (100, 37):
        a.step(n); b.step(n)
        assert np.array_equal(a.state(), b.state())
        assert np.array_equal(a.normc(), b.normc())
        assert a.conv() == b.conv()

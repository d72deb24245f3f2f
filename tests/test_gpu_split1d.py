"""1D lines too long for one block's shared memory (NX x M x bytes > 200 KB):
the four-step split N = N1 x N2 (row pass in Fourier space, column pass in
real space) against the CPU oracle, as for the other parity tests: states
1e-11 relative per step batch, observables 1e-10 (FP64), 2e-5 (FP32)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import case_id, case_params, initial_state, oracle_kwargs, rel_err

pytestmark = pytest.mark.gpu

CASES = [((1, 2, 1, (4096,)), "fp64", False), ((1, 2, 0, (4096,)), "fp64", False),
         ((1, 1, 1, (6000,)), "fp64", False), ((1, 1, 1, (4096,)), "fp64", True),
         ((1, 2, 1, (8192,)), "fp32", False), ((1, 2, 1, (2048,)), "fp64-split", False)]


@pytest.fixture(scope="module")
def F():
    import fortress_b200 as F
    if not F.device_ok():
        pytest.fail("no usable sm_100 device / libfgpe.so not loaded")
    return F


@pytest.mark.parametrize("case,precision,no_soc", CASES,
                         ids=lambda v: case_id(v) if isinstance(v, tuple) else str(v))
def test_split_line_matches_oracle(F, case, precision, no_soc):
    p = case_params(case)
    p["d"] = (20.0 / case[3][0],)            # a 20-wide box, resolved at every size
    mag = 0.0
    if no_soc:
        p["gamma"] = (0.0,)
        mag = 0.2
    orc = O.Oracle(**oracle_kwargs(p))
    phi = initial_state(orc, 2)
    orc.set_state(phi)
    if no_soc:
        orc.set_mag(mag)
    kernels = "auto"
    if precision.endswith("-split"):          # a line that fits one block, split on request
        precision, kernels = precision[:-6], "split-1d"
    prop = F.Propagator(**p, precision=precision, mag=mag, kernels=kernels)
    prop.set_state(phi)
    if case[2]:
        orc.normt(); prop.normt()
    tol = 1e-11 if precision == "fp64" else 2e-5
    for batch in (1, 5):
        prev = orc.state()
        norm_o = orc.step(batch)
        prop.step(batch)
        assert rel_err(prop.state(), orc.state()) < tol
        assert np.allclose(prop.normc(), norm_o, rtol=10 * tol, atol=0)
        en_g, mu_g, mz_g, rms_g = prop.observables()
        en_o, mu_o, mz_o = orc.energy()
        assert abs(en_g - en_o) <= 10 * tol * abs(en_o)
        assert np.allclose(rms_g, orc.rad(), rtol=10 * tol, atol=0)
        if batch == 1 and precision == "fp64":
            c_o = orc.maxdiff(prev)
            assert abs(prop.conv() - c_o) <= 1e-9 * c_o + 1e-15


def test_split_line_refuses_unfused_transforms(F):
    p = case_params((1, 2, 1, (4096,)))
    prop = F.Propagator(**p)
    prop.set_state(np.ones((4096, 1, 1, 5), complex))
    with pytest.raises(F.FgpeError, match="split"):
        prop.FFT()
    prop.SE()                                  # pointwise operators still work

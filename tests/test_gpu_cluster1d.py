"""Long 1D lines on one thread-block cluster (k_cl1d) against the two-pass
split (k_r1d/k_c1d) and the oracle, through the C ABI.

The cluster kernel keeps the four-step layout in the cluster's shared memory
for a whole call; per element it does the arithmetic of the two passes, and
only the order of the NORMC sum differs.  FP64 bars: states 1e-11 relative to
the oracle and 1e-13 to the two-pass path, observables 1e-10; FP32: 2e-5.
"""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import oracle_kwargs, rel_err

pytestmark = pytest.mark.gpu

# spin, nx, imaginary time, precision
CASES = [
    (2, 2048, 1, "fp64"),     # the reference's published 1D spin-2 grid
    (1, 1024, 1, "fp64"),
    (2, 2048, 0, "fp64"),
    (1, 4096, 0, "fp64"),
    (2, 2048, 1, "fp32"),
    (1, 1024, 0, "fp32"),
]


def _params(spin, nx, imag, precision, kernels="auto"):
    tau = (200.0, -5.0, 0.0) if spin == 1 else (300.0, 10.0, -8.0)
    return dict(dim=1, spin=spin, n=(nx,), d=(20.0 / nx,), dt=1e-4 if imag else 5e-5, imag_time=imag,
                tau=tau, gamma=(0.5,), alpha=(1.0, 1.0, 1.0), precision=precision, kernels=kernels)


def _state(spin, nx, seed):
    x = (np.arange(nx) - nx // 2) * (20.0 / nx)
    rng = np.random.default_rng(seed)
    ms = 2 * spin + 1
    phi = np.stack([np.exp(-x ** 2 / 2.0) * (1 + 0.05 * rng.standard_normal(nx)) *
                    np.exp(1j * rng.uniform(-0.4, 0.4, nx)) for _ in range(ms)], axis=-1)
    return phi.reshape(nx, 1, 1, ms)


def _case_id(c):
    return f"spin{c[0]}-{c[1]}-{'im' if c[2] else 're'}-{c[3]}"


@pytest.mark.parametrize("case", CASES, ids=_case_id)
def test_cluster_matches_two_pass_and_oracle(case):
    import fortress_b200 as F
    spin, nx, imag, precision = case
    phi = _state(spin, nx, 3)
    a = F.Propagator(**_params(spin, nx, imag, precision, "cluster-1d"))    # one cluster
    b = F.Propagator(**_params(spin, nx, imag, precision, "split-1d"))      # two passes
    p = _params(spin, nx, imag, "fp64")
    p.pop("precision"); p.pop("kernels")
    orc = O.Oracle(**oracle_kwargs(p))
    try:
        for h in (a, b):
            h.set_state(phi)
        orc.set_state(phi)
        if imag:
            a.normt(); b.normt(); orc.normt()
        tol_o = 1e-11 if precision == "fp64" else 2e-5
        tol_s = 1e-13 if precision == "fp64" else 1e-5
        for batch in (1, 2, 9):                 # one step, the two-step snapshot case, a longer call
            prev = orc.state()
            norm_o = orc.step(batch)
            a.step(batch)
            b.step(batch)
            sa = a.state()
            assert rel_err(sa, b.state()) < tol_s
            assert rel_err(sa, orc.state()) < tol_o
            assert np.allclose(a.normc(), norm_o, rtol=10 * tol_o, atol=0)
            en_a, mu_a, mz_a, rms_a = a.observables()
            en_o, mu_o, mz_o = orc.energy()
            assert abs(en_a - en_o) <= 10 * tol_o * abs(en_o)
            assert np.allclose(rms_a, orc.rad(), rtol=10 * tol_o, atol=0)
            c_o = orc.maxdiff(prev) if batch == 1 else None
            if c_o is not None and precision == "fp64":
                assert abs(a.conv() - c_o) <= 1e-9 * c_o + 1e-15
            if batch > 1:
                assert abs(a.conv() - b.conv()) <= (1e-9 if precision == "fp64" else 1e-3) * b.conv() + 1e-15
    finally:
        a.close()
        b.close()


def test_cluster_is_the_default_for_the_published_grid_and_launches_once_per_call():
    import fortress_b200 as F
    a = F.Propagator(**_params(2, 2048, 1, "fp64"))
    b = F.Propagator(**_params(2, 2048, 1, "fp64", "split-1d"))
    try:
        phi = _state(2, 2048, 4)
        for h in (a, b):
            h.set_state(phi)
            h.step(1)
        la, lb = a.kernel_launches(), b.kernel_launches()
        a.step(40)
        b.step(40)
        assert a.kernel_launches() - la == 1          # one cluster launch for the call
        assert b.kernel_launches() - lb == 80         # two passes per step
    finally:
        a.close()
        b.close()


def test_forced_cluster_on_a_short_line_and_refusal():
    import fortress_b200 as F
    # 512 = 16 x 32 divides over the 8-CTA cluster
    phi = _state(2, 512, 5)
    a = F.Propagator(**_params(2, 512, 1, "fp64", "cluster-1d"))
    b = F.Propagator(**_params(2, 512, 1, "fp64", "split-1d"))
    try:
        for h in (a, b):
            h.set_state(phi)
            h.normt()
            h.step(7)
        assert rel_err(a.state(), b.state()) < 1e-13
    finally:
        a.close()
        b.close()
    # 1200 = 30 x 40: N1 is no multiple of 8, so the forced cluster is refused
    with pytest.raises(F.FgpeError):
        F.Propagator(**_params(2, 1200, 1, "fp64", "cluster-1d"))
    # and the default falls back to the two passes
    c = F.Propagator(**_params(2, 1200, 1, "fp64"))
    c.close()


def test_default_takes_the_two_passes_for_long_lines():
    import fortress_b200 as F
    # 4096 x 5 > 10240: the two passes are faster than 8 SMs
    a = F.Propagator(**_params(2, 4096, 1, "fp64"))
    try:
        a.set_state(_state(2, 4096, 6))
        a.step(1)
        l0 = a.kernel_launches()
        a.step(8)
        assert a.kernel_launches() - l0 == 16
    finally:
        a.close()

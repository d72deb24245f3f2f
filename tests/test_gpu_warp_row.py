"""Row pass with one warp per x row (FGPE_KERNELS_WARP_ROW; the automatic
choice for FP64) against the block row kernel (FGPE_KERNELS_BLOCK_ROW) and
the oracle: the same per-element arithmetic, so real-time
states are bitwise equal and imaginary-time states differ only through the
NORMC summation order; both follow the oracle at the parity bars."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.helpers import initial_state, oracle_kwargs, rel_err

pytestmark = pytest.mark.gpu

CASES = [
    (3, 1, 0, (256, 16, 12), "fp64"), (3, 1, 1, (256, 12, 16), "fp64"), (2, 1, 1, (192, 128), "fp64"),
    (2, 2, 0, (128, 96), "fp64"), (2, 1, 0, (512, 64), "fp32"), (3, 2, 1, (256, 16, 16), "fp32"),
]


def _params(dim, spin, imag, n, prec):
    d = {2: (0.2, 0.25), 3: (0.15, 0.6, 0.65)}[dim]
    tau = (200.0, -5.0, 0.0) if spin == 1 else (300.0, 10.0, -8.0)
    return dict(dim=dim, spin=spin, n=n, d=d, dt=1e-3 if imag else 5e-4, imag_time=imag, tau=tau,
                gamma=(0.5, 0.3, 0.4)[:dim], alpha=(1.0, 1.3, 1.7), precision=prec)


@pytest.mark.parametrize("case", CASES, ids=lambda c: f"{c[0]}d-spin{c[1]}-{'im' if c[2] else 're'}-"
                                                      f"{'x'.join(map(str, c[3]))}-{c[4]}")
def test_warp_row_matches_block_row_and_oracle(case):
    import fortress_b200 as F
    dim, spin, imag, n, prec = case
    p = _params(dim, spin, imag, n, prec)
    q = dict(p)
    q.pop("precision")
    orc = O.Oracle(**oracle_kwargs(q))
    phi = initial_state(orc, seed=5)
    orc.set_state(phi)
    a = F.Propagator(**p, kernels="block-row")
    b = F.Propagator(**p, kernels="warp-row")
    for x in (a, b):
        x.set_state(phi)
        x.step(6)
    sa, sb = a.state(), b.state()
    if not imag:
        assert np.array_equal(sa, sb)
    assert rel_err(sb, sa) <= (1e-13 if prec == "fp64" else 1e-6)
    assert np.allclose(b.normc(), a.normc(), rtol=1e-12 if prec == "fp64" else 1e-6, atol=0)
    orc.step(6)
    assert rel_err(sb, orc.state()) <= (1e-11 if prec == "fp64" else 2e-5)
    eb, ea = b.observables()[0], a.observables()[0]
    assert abs(eb - ea) <= (1e-12 if prec == "fp64" else 1e-6) * abs(ea)

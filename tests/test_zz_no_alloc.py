"""fgpe_normc_noalloc (NORMC without a handle or any allocation) against the
handle's NORMC (fgpe_norms) on the same states, through the C ABI.

Collected last on purpose: it must also pass after every other test has used
the library in the same process.
"""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

CASES = [
    # dim, spin, n, d
    (1, 2, (256,), (0.05,)),
    (2, 2, (64, 48), (0.2, 0.25)),
    (2, 1, (96, 40), (0.1, 0.3)),
    (3, 1, (32, 16, 24), (0.3, 0.4, 0.35)),
]


def _state(shape, ms, seed):
    rng = np.random.default_rng(seed)
    return rng.standard_normal(shape + (ms,)) + 1j * rng.standard_normal(shape + (ms,))


def _handle_norms(F, dim, spin, n, d, phi):
    prop = F.Propagator(dim=dim, spin=spin, n=n, d=d, dt=1e-3, imag_time=True, tau=(1.0, 0.1, 0.0))
    try:
        prop.set_state(phi)
        return prop.normc()
    finally:
        prop.close()


def _noalloc_norms(L, dim, spin, n, d, phi):
    ms = 2 * spin + 1
    flat = np.ascontiguousarray(phi.reshape(-1, order="F"))
    dev = torch.from_numpy(flat.view(np.float64)).cuda()
    out = torch.full((ms,), float("nan"), dtype=torch.float64, device="cuda")
    nn = list(n) + [1] * (3 - len(n))
    dd = list(d) + [1.0] * (3 - len(d))
    torch.cuda.synchronize()
    rc = L.fgpe_normc_noalloc(dim, spin, nn[0], nn[1], nn[2], dd[0], dd[1], dd[2],
                              ctypes.c_void_p(dev.data_ptr()), ctypes.c_void_p(out.data_ptr()),
                              ctypes.c_void_p(torch.cuda.current_stream().cuda_stream))
    assert rc == 0, L.fgpe_last_error(None)
    torch.cuda.synchronize()
    return out.cpu().numpy()


@pytest.mark.parametrize("dim,spin,n,d", CASES)
def test_noalloc_matches_handle_normc_twice(dim, spin, n, d):
    import fortress_b200 as F
    from fortress_b200 import _abi
    L = _abi.load()
    ms = 2 * spin + 1
    shape = tuple(n) + (1,) * (3 - len(n))
    for call, seed in enumerate((11, 12)):           # two calls in a row
        phi = _state(shape, ms, seed + 10 * dim + spin)
        want = _handle_norms(F, dim, spin, n, d, phi)
        got = _noalloc_norms(L, dim, spin, n, d, phi)
        np.testing.assert_allclose(got, want, rtol=1e-12, atol=0, err_msg=f"call {call + 1}")


def test_noalloc_rejects_oversize_grid():
    from fortress_b200 import _abi
    L = _abi.load()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda")
    # 512 x 512 lines x 5 components exceeds the fixed scratch; rejected on
    # the host before anything is launched
    rc = L.fgpe_normc_noalloc(3, 2, 64, 512, 512, 0.1, 0.1, 0.1, ctypes.c_void_p(buf.data_ptr()),
                              ctypes.c_void_p(buf.data_ptr()), None)
    assert rc == _abi.FGPE_E_ARG
    assert b"scratch" in L.fgpe_last_error(None)
    rc = L.fgpe_normc_noalloc(2, 1, 31, 16, 1, 0.1, 0.1, 0.1, ctypes.c_void_p(buf.data_ptr()),
                              ctypes.c_void_p(buf.data_ptr()), None)
    assert rc == _abi.FGPE_E_ARG            # odd-sized axis is not the reference's Simpson rule

"""Tensor-core dense layer (fno_dense_tc: tcgen05.mma with the accumulator in
tensor memory) against the same layer in FP64 numpy on BF16-rounded
operands."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CASES = [(70, 40, 1000, 0, 1), (70, 40, 1000, 1, 0), (128, 128, 4096, 0, 1), (6, 128, 2560, 0, 0),
         (128, 32, 8192, 0, 1), (32, 7, 777, 1, 1), (1, 1, 300, 0, 0)]


def _gelu(x):
    c = np.sqrt(2.0 / np.pi)
    return 0.5 * x * (1.0 + np.tanh(c * (x + 0.044715 * x ** 3)))


@pytest.mark.parametrize("M,K,n,transw,act", CASES)
def test_dense_tc_matches_numpy(M, K, n, transw, act):
    from fortress_b200 import fno as FN
    L = FN.lib()
    rng = np.random.default_rng(M * 1000 + K + n)
    W = rng.standard_normal((K, M) if transw else (M, K)).astype(np.float32) / np.sqrt(K)
    x = rng.standard_normal((K, n)).astype(np.float32)
    b = rng.standard_normal(M).astype(np.float32)
    wb = torch.tensor(W.ravel()).to(torch.bfloat16).cuda()
    xd = torch.tensor(x).cuda()
    bd = torch.tensor(b).cuda()
    z = torch.full((M, n), float("nan"), device="cuda")
    h = torch.full((M, n), float("nan"), device="cuda")
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.fno_dense_tc(ctypes.c_void_p(wb.data_ptr()), transw, ctypes.c_void_p(xd.data_ptr()),
                        ctypes.c_void_p(bd.data_ptr()), ctypes.c_void_p(z.data_ptr()), ctypes.c_void_p(h.data_ptr()),
                        M, K, n, act, ctypes.c_void_p(err.data_ptr()), st)
    assert rc == 0
    torch.cuda.synchronize()
    assert int(err.item()) == 0
    Wr = wb.float().cpu().numpy().astype(np.float64).reshape(W.shape)
    Wm = Wr.T if transw else Wr
    xr = xd.to(torch.bfloat16).float().cpu().numpy().astype(np.float64)
    want_z = Wm @ xr + b[:, None]
    want_h = _gelu(want_z) if act else want_z
    got_z, got_h = z.cpu().numpy(), h.cpu().numpy()
    scale = np.abs(want_z).max()
    assert np.abs(got_z - want_z).max() <= 1e-5 * scale * max(1, K / 16)
    assert np.abs(got_h - want_h).max() <= 1e-5 * scale * max(1, K / 16) + 1e-6


def test_dense_tc_rejects_bad_shapes():
    from fortress_b200 import fno as FN
    L = FN.lib()
    t = torch.zeros(16, device="cuda")
    e = torch.zeros(1, dtype=torch.int32, device="cuda")
    p = ctypes.c_void_p(t.data_ptr())
    assert L.fno_dense_tc(p, 0, p, None, p, None, 129, 8, 16, 0, ctypes.c_void_p(e.data_ptr()), None) != 0
    assert L.fno_dense_tc(p, 0, p, None, p, None, 8, 200, 16, 0, ctypes.c_void_p(e.data_ptr()), None) != 0

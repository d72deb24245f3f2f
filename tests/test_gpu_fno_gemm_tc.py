"""Tensor-core strided batched GEMM (fno_gemm_tc: tcgen05.mma, FP32 operands
split into BF16 head and tail, FP32 accumulation in tensor memory) against
a PyTorch FP64 product of the same FP32 operands.  The cases follow the
learned guess's spectral stages: a DFT matrix shared by every channel plane
(the folded tall GEMM, and the transposed one when the shared matrix is the
left operand), the per-mode channel mix with BF16 weights, the long-K weight
gradient, column-major operands with M and N past one tile, beta
accumulation, and ragged K and N ends of the float4 operand reads.  Bound: |C - C_ref| <= 1e-4 (|A| |B|) elementwise (the dropped
lo*lo term and the tail roundings are about 2^-16 of each product)."""
import ctypes

import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

# batch, M, N, K, A strides, B strides, C strides, a_bf16, alpha, beta
CASES = {
    "dft-shared-right": (64, 64, 16, 64, (64 * 64, 64, 1), (0, 16, 1), (64 * 16, 16, 1), 0, 1.0, 0.0),
    "dft-shared-left": (48, 32, 16, 128, (0, 128, 1), (128 * 16, 16, 1), (32 * 16, 16, 1), 0, 1.0, 0.0),
    "mode-mix-bf16": (40, 64, 24, 64, (64 * 64, 64, 1), (64 * 24, 24, 1), (64 * 24, 24, 1), 1, 0.5, 1.0),
    "weight-grad-long-k": (4, 32, 40, 2048, (2048, 8192, 1), (2048, 1, 8192), (32 * 40, 40, 1), 0, 1.0, 0.0),
    "column-major-two-tiles": (1, 200, 300, 70, (0, 1, 200), (0, 300, 1), (0, 1, 200), 0, 1.0, 0.0),
    "interleaved-output": (16, 64, 64, 16, (64 * 16 * 2, 16, 1), (0, 64, 1), (64 * 64, 64, 1), 0, 1.0 / 4096, 1.0),
    "one-element": (1, 1, 1, 1, (0, 1, 1), (0, 1, 1), (0, 1, 1), 0, 2.0, 0.0),
    "ragged-k-vectors": (3, 50, 20, 70, (50 * 72, 72, 1), (0, 20, 1), (50 * 20, 20, 1), 0, 1.0, 0.0),
    "ragged-k-along-k": (2, 40, 36, 70, (40 * 72, 72, 1), (72 * 36, 1, 72), (40 * 36, 36, 1), 0, 1.0, 0.0),
}


def _span(batch, rows, cols, s):
    return 1 + (batch - 1) * s[0] + (rows - 1) * s[1] + (cols - 1) * s[2]


@pytest.mark.parametrize("name", list(CASES))
def test_gemm_tc_matches_fp64(name):
    from fortress_b200 import fno as FN
    L = FN.lib()
    batch, M, N, K, sA, sB, sC, a_bf16, alpha, beta = CASES[name]
    rng = np.random.default_rng(len(name) * 7919 + M)
    a = torch.tensor(rng.standard_normal(_span(batch, M, K, sA)).astype(np.float32))
    b = torch.tensor(rng.standard_normal(_span(batch, K, N, sB)).astype(np.float32))
    c = torch.tensor(rng.standard_normal(_span(batch, M, N, sC)).astype(np.float32))
    if a_bf16:
        a = a.to(torch.bfloat16)
    A = torch.as_strided(a.double(), (batch, M, K), sA)
    B = torch.as_strided(b.double(), (batch, K, N), sB)
    C0 = torch.as_strided(c.double(), (batch, M, N), sC)
    want = alpha * torch.bmm(A, B) + beta * C0
    bound = 1e-4 * torch.bmm(A.abs(), B.abs()) * abs(alpha) + 1e-6 * (beta * C0).abs()
    ad, bd, cd = a.cuda(), b.cuda(), c.cuda()
    err = torch.zeros(1, dtype=torch.int32, device="cuda")
    st = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    rc = L.fno_gemm_tc(batch, M, N, K, alpha, ctypes.c_void_p(ad.data_ptr()), a_bf16, *sA,
                       ctypes.c_void_p(bd.data_ptr()), *sB, beta, ctypes.c_void_p(cd.data_ptr()), *sC,
                       ctypes.c_void_p(err.data_ptr()), st)
    assert rc == 0
    torch.cuda.synchronize()
    assert err.item() == 0
    got = torch.as_strided(cd.cpu().double(), (batch, M, N), sC)
    # entries of the buffer outside C stay untouched
    mask = torch.zeros(cd.numel(), dtype=torch.bool)
    torch.as_strided(mask, (batch, M, N), sC).fill_(True)
    assert torch.equal(cd.cpu()[~mask], c[~mask])
    excess = ((got - want).abs() - bound).max().item()
    assert excess <= 0.0, (name, excess)


def test_gemm_tc_matches_the_fp32_gemm_in_the_network():
    """One forward and backward of the 2D network with every GEMM on
    fno_gemm_tc and on the SIMT FP32 fno_gemm (the BF16 dense-layer kernel
    off in both): outputs and gradients agree to the split-BF16 precision."""
    from fortress_b200 import fno as FN
    rng = np.random.default_rng(3)
    p = FN.init_params(width=16, modes=8, layers=2, hidden=32, seed=4)
    a = FN.input_channels(rng.uniform(-1, 1, (4, 5)), 32)
    tgt = torch.randn(6, 4 * 32 * 32, device="cuda", generator=torch.Generator("cuda").manual_seed(2))
    outs = []
    for tc in (False, True):
        net = FN.FNO(32, 4, params=p, width=16, modes=8, layers=2, hidden=32, tensor_cores=tc)
        net._use_tc = lambda M, K: False          # dense layers through the GEMM entry point
        net.forward(a)
        net.loss(tgt)
        net.backward()
        torch.cuda.synchronize()
        assert not net.tc_error()
        outs.append((net.out.clone(), {k: v.clone() for k, v in net.g.items()}))
    (o0, g0), (o1, g1) = outs
    assert (o1 - o0).abs().max().item() <= 1e-4 * o0.abs().max().item()
    for k in g0:
        assert (g1[k] - g0[k]).abs().max().item() <= 1e-3 * g0[k].abs().max().item() + 1e-12, k

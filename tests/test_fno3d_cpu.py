"""Index arithmetic of the 3D learned-guess network's spectral layer, on the
CPU: the chain of strided batched GEMMs in fortress_b200/fno3d.py (forward
and backward) is run with an as_strided emulation of fno_gemm's contract
(include/fno.h) and compared with the FP64 numpy oracle's 3D spectral
convolution and its adjoint (oracle/fno_oracle.py)."""
import numpy as np
import pytest

from oracle import fno_oracle as FO

torch = pytest.importorskip("torch")


def _gemm_emulated(self, batch, M, N, K, A, sA, B_, sB, C, sC, alpha=1.0, beta=0.0, a_bf16=False, aoff=0, boff=0,
                   coff=0):
    """C[b](i,j) = alpha sum_k A[b](i,k) B[b](k,j) + beta C[b](i,j), elements
    addressed as in fno_gemm."""
    a = torch.as_strided(A.reshape(-1), (batch, M, K), sA, aoff).double()
    b = torch.as_strided(B_.reshape(-1), (batch, K, N), sB, boff).double()
    c = torch.as_strided(C.reshape(-1), (batch, M, N), sC, coff)
    c.copy_((alpha * torch.bmm(a, b) + beta * c.double()).to(c.dtype))


def _net(n, B, W, M, seed):
    from fortress_b200 import fno3d as F3
    net = object.__new__(F3.FNO3)
    net.torch = torch
    net.n, net.B, net.W, net.M, net.F = n, B, W, M, 2 * M
    net.S, net.NMODE, net.layers, net.train, net.dev = n ** 3, 4 * M * M * M, 1, True, "cpu"
    net.mat_dtype = torch.float64
    net._dft()
    CB, FM = W * B, 2 * M * M
    z = lambda k: torch.zeros(k, dtype=torch.float64)
    net.T1, net.U2 = z(CB * n * 2 * n * M), z(CB * n * 2 * n * M)
    net.T2, net.U1 = z(CB * n * 2 * FM), z(CB * n * 2 * FM)
    net.Hm, net.Gm, net.dHm = [z(net.NMODE * 2 * CB)], z(net.NMODE * 2 * CB), z(net.NMODE * 2 * CB)
    rng = np.random.default_rng(seed)
    Rr = rng.standard_normal((W, W, 2 * M, 2 * M, M))
    Ri = rng.standard_normal((W, W, 2 * M, 2 * M, M))
    dev = F3.FNO3._to_device_layout({"Rr0": Rr, "Ri0": Ri})
    rr, ri = dev["Rr0"], dev["Ri0"]
    big = np.block([[rr, -ri], [ri, rr]])                       # [mode][2O][2C]
    net.pb = {"Rbig0": torch.tensor(big.reshape(-1))}
    net.g_rbig = z(net.NMODE * 4 * W * W)
    net.g = {"Rr0": z(net.NMODE * W * W), "Ri0": z(net.NMODE * W * W)}

    def fold(l):
        g = net.g_rbig.reshape(net.NMODE, 2 * W, 2 * W)
        net.g["Rr0"].copy_((g[:, :W, :W] + g[:, W:, W:]).reshape(-1))
        net.g["Ri0"].copy_((g[:, W:, :W] - g[:, :W, W:]).reshape(-1))

    net._rbig_fold = fold
    net.gemm = _gemm_emulated.__get__(net)
    return net, Rr, Ri


@pytest.mark.parametrize("n,B,W,M", [(8, 2, 3, 2), (12, 1, 2, 3)])
def test_spectral_chain_matches_oracle(n, B, W, M):
    net, Rr, Ri = _net(n, B, W, M, seed=n)
    rng = np.random.default_rng(1)
    h = rng.standard_normal((W, B, n, n, n))                    # device layout [C][B][Z][Y][X]
    zt = torch.zeros(W * B * n ** 3, dtype=torch.float64)
    net.spectral(0, torch.tensor(h.reshape(-1)), zt)
    Ef, Eh, w = FO.dft_mats3(n, M)
    K, H = FO.spectral3(np.transpose(h, (1, 0, 2, 3, 4)), Rr, Ri, Ef, Eh, w)
    got = np.transpose(zt.numpy().reshape(W, B, n, n, n), (1, 0, 2, 3, 4))
    assert np.abs(got - K).max() <= 1e-12 * np.abs(K).max()
    # adjoint: dh and the R gradients
    dK = rng.standard_normal((B, W, n, n, n))
    dh = torch.zeros(W * B * n ** 3, dtype=torch.float64)
    net.spectral_bwd(0, torch.tensor(np.transpose(dK, (1, 0, 2, 3, 4)).reshape(-1).copy()), dh)
    dh_o, gRr, gRi = FO.spectral3_bwd(dK, H, Rr, Ri, Ef, Eh, w)
    got = np.transpose(dh.numpy().reshape(W, B, n, n, n), (1, 0, 2, 3, 4))
    assert np.abs(got - dh_o).max() <= 1e-12 * np.abs(dh_o).max()
    g = net.g["Rr0"].numpy().reshape(2 * M, 2 * M, M, W, W)
    assert np.abs(np.transpose(g, (3, 4, 0, 1, 2)) - gRr).max() <= 1e-12 * np.abs(gRr).max()
    g = net.g["Ri0"].numpy().reshape(2 * M, 2 * M, M, W, W)
    assert np.abs(np.transpose(g, (3, 4, 0, 1, 2)) - gRi).max() <= 1e-12 * np.abs(gRi).max()

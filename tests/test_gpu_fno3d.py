"""3D learned-guess network on the device (fortress_b200.fno3d, kernels of
include/fno.h) against the FP64 numpy oracle (oracle/fno_oracle.py, 3D form):
forward values, loss and every parameter gradient, on the FP32 GEMM path and
on the tcgen05 dense layers."""
import numpy as np
import pytest

from oracle import fno_oracle as FO

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CFG = dict(width=6, modes=3, layers=2, hidden=12)


def _bf16(x):
    return torch.tensor(np.asarray(x), dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()


def _setup(n=12, B=2, seed=1, tc=True):
    from fortress_b200 import fno3d as F3
    p = F3.init_params(cin=7, cout=6, seed=seed, **CFG)
    rng = np.random.default_rng(seed + 100)
    for k in p:
        if k.startswith(("b", "c")):
            p[k] = 0.1 * rng.standard_normal(p[k].shape)
    pn = rng.uniform(-1, 1, size=(B, 4))
    a = F3.input_channels(pn, n)
    tgt = rng.standard_normal((6, B, n, n, n)).astype(np.float32)
    net = F3.FNO3(n, B, params=p, cin=7, cout=6, tensor_cores=tc, **CFG)
    po = {k: (_bf16(v) if (k[0] in "PQW" or k.startswith("R")) else v) for k, v in p.items()}
    return net, po, a, tgt


# (tensor cores, output / loss / gradient tolerance relative to the largest
# entry), as for the 2D network: FP32 GEMMs follow the FP64 oracle closely,
# the tcgen05 path rounds the dense layers' activations to BF16.
TOL = {False: (1e-4, 1e-5, 1e-3), True: (1e-2, 1e-2, 5e-2)}


@pytest.mark.parametrize("tc", [False, True], ids=["fp32-gemm", "tcgen05"])
def test_forward_loss_and_gradients_match_oracle(tc):
    net, po, a, tgt = _setup(tc=tc)
    t_out, t_loss, t_grad = TOL[tc]
    a_o = np.transpose(a.astype(np.float64), (1, 0, 2, 3, 4))
    t_o = np.transpose(tgt.astype(np.float64), (1, 0, 2, 3, 4))
    out_o = FO.forward3(po, a_o, modes=CFG["modes"], layers=CFG["layers"])
    loss_o, g_o = FO.loss_and_grad3(po, a_o, t_o, modes=CFG["modes"], layers=CFG["layers"])
    out = net.forward(a).cpu().numpy().reshape((6,) + out_o.shape[:1] + out_o.shape[2:])
    out = np.transpose(out, (1, 0, 2, 3, 4))
    assert np.abs(out - out_o).max() <= t_out * np.abs(out_o).max()
    loss = float(net.loss(torch.tensor(tgt.reshape(6, -1), device="cuda")).item())
    assert abs(loss - loss_o) <= t_loss * abs(loss_o)
    net.backward()
    torch.cuda.synchronize()
    assert not net.tc_error()
    g = net.grads_numpy()
    assert set(g) == set(g_o)
    for k in g_o:
        err = np.abs(g[k] - g_o[k]).max()
        scale = np.abs(g_o[k]).max()
        assert err <= t_grad * scale + 1e-9, (k, err, scale)


def test_spinor_layout_and_resolution_change():
    """spinor() returns PHI(NX,NY,NZ,3); the same parameters evaluate on a
    finer grid (only the truncated DFT matrices change)."""
    from fortress_b200 import fno3d as F3
    net, po, a, tgt = _setup(n=12, B=1)
    net.forward(a)
    phi = net.spinor(0)
    o = net.out.reshape(6, 12, 12, 12).double().cpu().numpy()
    assert phi.shape == (12, 12, 12, 3)
    assert phi[3, 5, 7, 1] == pytest.approx(o[2, 7, 5, 3] + 1j * o[3, 7, 5, 3], rel=1e-12)
    fine = F3.FNO3(24, 1, params=net.params_numpy(), cin=7, cout=6, train=False, **CFG)
    fine.forward(F3.input_channels(np.zeros((1, 4)), 24))
    assert np.all(np.isfinite(fine.spinor(0)))

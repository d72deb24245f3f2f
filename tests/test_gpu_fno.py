"""Learned-guess network on the device (fortress_b200.fno, kernels of
include/fno.h) against the FP64 numpy oracle (oracle/fno_oracle.py): forward
values, loss, every parameter gradient, one Adam step, and a short training
run that must lower the loss."""
import numpy as np
import pytest

from oracle import fno_oracle as FO

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

CFG = dict(width=8, modes=4, layers=2, hidden=16)


def _bf16(x):
    return torch.tensor(np.asarray(x), dtype=torch.float32).to(torch.bfloat16).to(torch.float64).numpy()


def _setup(n=16, B=2, seed=1, tc=True):
    from fortress_b200 import fno as FN
    p = FN.init_params(cin=7, cout=6, seed=seed, **CFG)
    rng = np.random.default_rng(seed + 100)
    for k in p:                       # non-zero biases so their gradients are exercised
        if k.startswith(("b", "c")):
            p[k] = 0.1 * rng.standard_normal(p[k].shape)
    pn = rng.uniform(-1, 1, size=(B, 5))
    a = FN.input_channels(pn, n)
    tgt = rng.standard_normal((6, B, n, n)).astype(np.float32)
    net = FN.FNO(n, B, params=p, cin=7, cout=6, tensor_cores=tc, **CFG)
    # the oracle sees the weights the GEMMs read: BF16-rounded matrices
    po = {k: (_bf16(v) if (k[0] in "PQW" or k.startswith("R")) else v) for k, v in p.items()}
    return FN, net, po, a, tgt


def _oracle(po, a, tgt):
    a_o = np.transpose(a.astype(np.float64), (1, 0, 2, 3))            # [B][7][n][n]
    t_o = np.transpose(tgt.astype(np.float64), (1, 0, 2, 3))
    out = FO.forward(po, a_o, modes=CFG["modes"], layers=CFG["layers"])
    loss, g = FO.loss_and_grad(po, a_o, t_o, modes=CFG["modes"], layers=CFG["layers"])
    return np.transpose(out, (1, 0, 2, 3)), loss, g


# (tensor cores, output / loss / gradient tolerance relative to the largest
# entry): the FP32 GEMM path follows the FP64 oracle closely; the tcgen05 path
# also rounds the activations entering each dense layer to BF16 (8 bits).
TOL = {False: (1e-4, 1e-5, 1e-3), True: (1e-2, 1e-2, 5e-2)}


@pytest.mark.parametrize("tc", [False, True], ids=["fp32-gemm", "tcgen05"])
def test_forward_loss_and_gradients_match_oracle(tc):
    FN, net, po, a, tgt = _setup(tc=tc)
    t_out, t_loss, t_grad = TOL[tc]
    out_o, loss_o, g_o = _oracle(po, a, tgt)
    t_dev = torch.tensor(tgt.reshape(6, -1), device="cuda")
    out = net.forward(a).cpu().numpy().reshape(out_o.shape)
    assert np.abs(out - out_o).max() <= t_out * np.abs(out_o).max()
    loss = float(net.loss(t_dev).item())
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


def test_adam_step_matches_formula():
    FN, net, po, a, tgt = _setup(seed=3)
    t_dev = torch.tensor(tgt.reshape(6, -1), device="cuda")
    net.forward(a); net.loss(t_dev); net.backward()
    w0 = {k: v.detach().cpu().numpy().copy() for k, v in net.p.items()}
    g = {k: v.detach().cpu().numpy().copy() for k, v in net.g.items()}
    net.adam(lr=1e-2)
    torch.cuda.synchronize()
    for k in w0:
        m = 0.1 * g[k]
        v = 0.001 * g[k] ** 2
        want = w0[k] - 1e-2 * (m / 0.1) / (np.sqrt(v / 0.001) + 1e-8)
        np.testing.assert_allclose(net.p[k].cpu().numpy(), want, rtol=1e-5, atol=1e-6, err_msg=k)
    # the BF16 copies follow the master weights
    np.testing.assert_allclose(net.pb["Q1"].float().cpu().numpy(), net.p["Q1"].cpu().numpy().ravel(),
                               rtol=1e-2, atol=1e-3)


def test_training_lowers_the_loss():
    FN, net, po, a, tgt = _setup(n=32, B=4, seed=5)
    # a learnable target: a smooth function of the inputs
    x = a[5]; y = a[6]
    tgt = np.stack([np.exp(-(x ** 2 + y ** 2) * 4) * (1 + 0.3 * a[q % 5]) for q in range(6)]).astype(np.float32)
    t_dev = torch.tensor(tgt.reshape(6, -1), device="cuda")
    net.forward(a)
    first = float(net.loss(t_dev).item())
    for _ in range(60):
        net.forward()
        net.loss(t_dev)
        net.backward()
        net.adam(lr=3e-3)
    net.forward()
    last = float(net.loss(t_dev).item())
    assert last < 0.3 * first, (first, last)

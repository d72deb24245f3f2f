"""The numpy FNO restatement: analytic gradients against central finite
differences, and the spectral layer against numpy's FFT definition."""
import numpy as np
import pytest

from oracle import fno_oracle as FO


def _small():
    rng = np.random.default_rng(1)
    p = FO.init_params(width=6, modes=3, layers=2, hidden=8, seed=2)
    for k in p:
        if k.startswith("b") or k.startswith("c"):
            p[k] = 0.1 * rng.standard_normal(p[k].shape)
        if k.startswith("R"):
            p[k] = p[k] * 20
    a = rng.standard_normal((2, 7, 12, 12))
    t = rng.standard_normal((2, 6, 12, 12))
    return p, a, t


def test_spectral_layer_matches_fft_definition():
    rng = np.random.default_rng(0)
    n, m, c = 16, 4, 3
    h = rng.standard_normal((1, c, n, n))
    Ex, Ey, w = FO.dft_mats(n, m)
    R = np.zeros((c, c, 2 * m, m)); Ri = np.zeros_like(R)
    for i in range(c):
        R[i, i] = 1.0                      # identity mixing: K = low-pass of h
    K, H = FO.spectral(h, R, Ri, Ex, Ey, w)
    Hf = np.fft.fft2(h[0], axes=(1, 2))
    kx = np.concatenate([np.arange(m), np.arange(n - m, n)])
    assert np.allclose(H[0], Hf[:, kx][:, :, :m])
    # low-pass reconstruction through the real inverse FFT with Hermitian fill
    Z = np.zeros((c, n, n // 2 + 1), complex)
    Z[:, kx, :m] = Hf[:, kx][:, :, :m]
    ref = np.fft.irfft2(Z, s=(n, n), axes=(1, 2))
    # irfft2 keeps the real part of the ky=0 column and doubles ky>0: the
    # same real operator as Re(sum_k w_k Z_k e^{ik.x}) / N^2
    assert np.allclose(K[0], ref, atol=1e-12)


@pytest.mark.parametrize("name", ["P", "bP", "W0", "b1", "Rr0", "Ri1", "Q1", "c1", "Q2", "c2"])
def test_gradients_finite_differences(name):
    p, a, t = _small()
    loss, g = FO.loss_and_grad(p, a, t, modes=3, layers=2)
    rng = np.random.default_rng(3)
    flat = p[name].reshape(-1)
    idx = rng.choice(flat.size, size=min(6, flat.size), replace=False)
    for i in idx:
        old = flat[i]
        eps = 1e-6
        flat[i] = old + eps; lp = FO.loss_and_grad(p, a, t, modes=3, layers=2)[0]
        flat[i] = old - eps; lm = FO.loss_and_grad(p, a, t, modes=3, layers=2)[0]
        flat[i] = old
        fd = (lp - lm) / (2 * eps)
        an = g[name].reshape(-1)[i]
        assert abs(fd - an) <= 1e-6 * max(1.0, abs(fd)) + 1e-9, (name, i, fd, an)

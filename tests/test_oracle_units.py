"""Unit checks of the oracle's building blocks against independent CPU
implementations (numpy FFT, scipy zheev, analytic identities)."""
import numpy as np
import pytest

from oracle import oracle as O


@pytest.mark.parametrize("n", [8, 16, 96, 128, 192, 250, 256, 384, 512, 1024])
def test_fft_matches_numpy(n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x)
    assert np.abs(O.fft1d(x, -1) - ref).max() <= 1e-14 * np.abs(ref).max()
    assert np.abs(O.fft1d(x, +1) - np.fft.ifft(x) * n).max() <= 1e-14 * np.abs(ref).max()


@pytest.mark.parametrize("n", [8, 10, 64, 2048])
def test_simpson_weights(n):
    # the composite rule integrates cubics exactly
    dx = 0.1
    x = np.arange(n) * dx
    f = 1 + 2 * x - x ** 2 + 0.5 * x ** 3
    L = x[-1]
    exact = L + L ** 2 - L ** 3 / 3 + 0.5 * L ** 4 / 4
    assert abs(O.simpson(f, dx) - exact) < 1e-9 * max(1, abs(exact))


def test_diff_stencils():
    n, dx = 64, 0.05
    x = np.arange(n) * dx
    p = np.sin(2 * np.pi * x / (n * dx))  # periodic: the wrapped edges are exact too
    d = O.diff(p, dx)
    ex = 2 * np.pi / (n * dx) * np.cos(2 * np.pi * x / (n * dx))
    assert np.abs(d[4:-4] - ex[4:-4]).max() < 1e-9
    assert np.abs(d - ex).max() < 2e-5


def test_spin2_exponential_matches_zheev():
    sl = pytest.importorskip("scipy.linalg.lapack")
    rng = np.random.default_rng(7)
    for trial in range(50):
        c = (rng.standard_normal(6) + 1j * rng.standard_normal(6)) * 10 ** rng.uniform(-3, 2)
        v = rng.standard_normal(5) + 1j * rng.standard_normal(5)
        for cdt in (-1j * 1e-3, 1e-3, -1j * 0.05):
            H = np.zeros((5, 5), complex)
            for (r, q), val in zip([(0, 1), (0, 2), (1, 2), (2, 3), (2, 4), (3, 4)], c):
                H[r, q] = val
                H[q, r] = np.conj(val)
            w, V, info = sl.zheev(H, compute_v=1, lower=1)
            assert info == 0
            ref = V @ (np.exp(-1j * cdt * w) * (V.conj().T @ v))
            ours = O.expm_se2(c, cdt, v)
            assert np.abs(ours - ref).max() <= 1e-13 * max(1.0, np.abs(ref).max())


def test_real_time_conserves_norm():
    kw = dict(dim=2, spin=1, nx=32, ny=32, dx=0.25, dy=0.25, dt=1e-3, imag=0,
              tau=(50.0, -2.0, 0.0), gx=0.7, gy=0.4)
    o = O.Oracle(**kw)
    o.initialize()
    # every sub-step is unitary, so the plain l2 sum is conserved (the
    # Simpson-weighted NORMC is not exactly)
    n0 = np.sum(np.abs(o.state()) ** 2)
    o.step(20)
    assert abs(np.sum(np.abs(o.state()) ** 2) - n0) < 1e-12 * n0


def test_harmonic_ground_state_energy():
    # tau = 0, gamma = 0: ground state of -d2/dx2 + x^2 (units of the
    # reference, energy printed /2) is E/2 = 1/2 per dimension.
    kw = dict(dim=1, spin=1, nx=256, dx=0.1, dt=5e-4, imag=1, tau=(0.0, 0.0, 0.0))
    o = O.Oracle(**kw)
    o.initialize()
    o.normt()
    o.step(4000)
    en, mu, mz = o.energy()
    assert abs(en / 2 - 0.5) < 1e-6

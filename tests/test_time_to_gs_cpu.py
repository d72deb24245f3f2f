"""Host logic of the time-to-ground-state experiment, on the CPU: the
spectral prolongation's zero padding (with numpy's FFT standing in for the
library's transforms) reproduces a band-limited function on the fine grid,
and the "for good" rule of the time measurement."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")


def test_pad_spectrum_interpolates_band_limited_functions():
    from fortress_b200.experiments import time_to_gs as T
    m, n, L = 8, 16, 25.6
    rng = np.random.default_rng(0)
    coef = rng.standard_normal((3, 3, 3)) + 1j * rng.standard_normal((3, 3, 3))

    def f(k):
        x = (-1.0 + 2.0 * np.arange(k) / k) * L / 2
        out = np.zeros((k, k, k), complex)
        for a in range(3):
            for b in range(3):
                for c in range(3):
                    kz, ky, kx = (a - 1, b - 1, c - 1)
                    out += coef[a, b, c] * np.exp(2j * np.pi * (kz * x[:, None, None] + ky * x[None, :, None]
                                                                + kx * x[None, None, :]) / L)
        return out

    coarse = np.stack([f(m)] * 3)
    spec = torch.tensor(np.fft.fftn(coarse, axes=(1, 2, 3)))
    big = T.pad_spectrum(spec, n).numpy()
    fine = np.fft.ifftn(big, axes=(1, 2, 3)) * (n / m) ** 3
    assert np.abs(fine - np.stack([f(n)] * 3)).max() < 1e-12 * np.abs(fine).max()


def test_time_to_counts_from_the_last_entry_into_the_band():
    from fortress_b200.experiments import time_to_gs as T
    e_star = 10.0
    tr = [("fp32", 100, 1.0, 10.1, 0, 0), ("fp64", 100, 2.0, 10.0 + 5e-8, 0, 0),
          ("fp64", 200, 3.0, 10.0 + 2e-7, 0, 0), ("fp64", 300, 4.0, 10.0 + 5e-8, 0, 0),
          ("fp64", 400, 5.0, 10.0 + 1e-8, 0, 0)]
    steps, wall = T.time_to(tr, e_star)
    assert wall == 4.0 and steps == {"fp32": 100, "fp64": 300}
    assert T.time_to(tr[:3], e_star) is None

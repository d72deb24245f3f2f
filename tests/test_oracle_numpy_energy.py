"""The C oracle's 2D observables against the numpy restatement, from
cgpe2d.f90: ENERGY 1075-1281 (spin-1 and spin-2 with the SO-coupling terms),
RAD 1032-1070, FXYZ 891-913, MAT_C 919-942, and DIFF (diff.f90:4-33) with
its 1-based indices shifted by one.  Energy, chemical potentials,
magnetisation and rms sizes of a generic complex spinor."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.test_oracle_numpy_2d import EPS, S15, _mat_c, _spin_matrices
from tests.test_oracle_numpy_projection import np_normc, np_simpson


def np_diff(p, dx):
    n = len(p)

    def P(i):                    # the reference's P(i), 1-based
        return p[i - 1]

    d = np.empty(n)
    d[0] = (P(n - 1) - 8.0 * P(n) + 8.0 * P(2) - P(3)) / (12.0 * dx)
    d[1] = (P(n) - 8.0 * P(1) + 8.0 * P(3) - P(4)) / (12.0 * dx)
    for i in (3, 4, n - 3, n - 2):
        d[i - 1] = (P(i - 2) - 8.0 * P(i - 1) + 8.0 * P(i + 1) - P(i + 2)) / (12.0 * dx)
    for i in range(5, n - 3):
        d[i - 1] = (3.0 * P(i - 4) - 32.0 * P(i - 3) + 168.0 * P(i - 2) - 672.0 * P(i - 1) +
                    672.0 * P(i + 1) - 168.0 * P(i + 2) + 32.0 * P(i + 3) - 3.0 * P(i + 4)) / (840.0 * dx)
    d[n - 2] = (P(n - 3) - 8.0 * P(n - 2) + 8.0 * P(n) - P(1)) / (12.0 * dx)
    d[n - 1] = (P(n - 2) - 8.0 * P(n - 1) + 8.0 * P(1) - P(2)) / (12.0 * dx)
    return d


def _derivatives(phi, dx, dy):
    nx, ny, ms = phi.shape
    dpx = np.empty(phi.shape, complex)
    dpy = np.empty(phi.shape, complex)
    for k in range(ms):
        for j in range(ny):
            dpx[:, j, k] = np_diff(phi[:, j, k].real, dx) + 1j * np_diff(phi[:, j, k].imag, dx)
        for i in range(nx):
            dpy[i, :, k] = np_diff(phi[i, :, k].real, dy) + 1j * np_diff(phi[i, :, k].imag, dy)
    return dpx, dpy


def _integrate(f, dx, dy):
    return np_simpson(np.array([np_simpson(f[:, j], dx) for j in range(f.shape[1])]), dy)


def np_energy(phi, x, y, kw):
    spin, dx, dy = kw["spin"], kw["dx"], kw["dy"]
    t0, t1, t2 = kw["tau"]
    gx, gy = kw["gx"], kw["gy"]
    v = kw["ax"] ** 2 * x[:, None] ** 2 + kw["ay"] ** 2 * y[None, :] ** 2
    sx, sy = _spin_matrices(spin)
    sz = np.arange(spin, -spin - 1, -1, dtype=float)
    fx = np.real(np.einsum("...i,ij,...j->...", phi.conj(), sx, phi))
    fy = np.real(np.einsum("...i,ij,...j->...", phi.conj(), sy, phi))
    a = np.abs(phi) ** 2
    fz = (a * sz).sum(-1)
    rho = a.sum(-1)
    dpx, dpy = _derivatives(phi, dx, dy)
    dp2 = np.abs(dpx) ** 2 + np.abs(dpy) ** 2
    p = [phi[..., m] for m in range(2 * spin + 1)]
    c = [u.conj() for u in p]
    X = [dpx[..., m] for m in range(2 * spin + 1)]
    Y = [dpy[..., m] for m in range(2 * spin + 1)]
    ci = 1j
    if spin == 1:
        r2 = np.sqrt(2.0)
        t = [v * rho + t0 * rho ** 2 / 2.0 + t1 * (fx ** 2 + fy ** 2 + fz ** 2) / 2.0 + dp2.sum(-1) +
             r2 * (c[0] * (-ci * gx * X[1] - gy * Y[1]) + c[1] * (-ci * gx * X[2] - gy * Y[2]) +
                   c[1] * (-ci * gx * X[0] + gy * Y[0]) + c[2] * (-ci * gx * X[1] + gy * Y[1])),
             a[..., 0] - a[..., 2],
             v * a[..., 0] + dp2[..., 0] + t0 * rho * a[..., 0] + t1 * (a[..., 0] + a[..., 1] - a[..., 2]) * a[..., 0] +
             t1 * c[2] * p[1] ** 2 * c[0] + r2 * (c[0] * (-ci * gx * X[1] - gy * Y[1])),
             v * a[..., 1] + dp2[..., 1] + t0 * rho * a[..., 1] + t1 * (a[..., 0] + a[..., 2]) * a[..., 1] +
             2.0 * t1 * p[0] * p[2] * c[1] ** 2 +
             r2 * (c[1] * (-ci * gx * X[2] - gy * Y[2]) + c[1] * (-ci * gx * X[0] + gy * Y[0])),
             v * a[..., 2] + dp2[..., 2] + t0 * rho * a[..., 2] + t1 * (a[..., 1] + a[..., 2] - a[..., 0]) * a[..., 2] +
             t1 * c[0] * p[1] ** 2 * c[2] + r2 * (c[2] * (-ci * gx * X[1] + gy * Y[1]))]
    else:
        c12, c13, c23, c34, c35, c45 = _mat_c(phi, kw["tau"])
        theta = (2.0 * p[0] * p[4] - 2.0 * p[1] * p[3] + p[2] ** 2) / np.sqrt(5.0)
        t = [v * rho + t0 * rho ** 2 / 2.0 + t1 * (fx ** 2 + fy ** 2 + fz ** 2) / 2.0 +
             t2 * (theta * theta.conj()) / 2.0 + dp2.sum(-1)
             - ci * 2.0 * (c[0] * gx * X[1] - ci * c[0] * gy * Y[1] + c[1] * gx * X[0] + ci * c[1] * gy * Y[0] +
                           S15 * (c[1] * gx * X[2] - ci * c[1] * gy * Y[2] + c[2] * gx * X[1] +
                                  ci * c[2] * gy * Y[1] + c[2] * gx * X[3] - ci * c[2] * gy * Y[3] +
                                  c[3] * gx * X[2] + ci * c[3] * gy * Y[2]) +
                           c[3] * gx * X[4] - ci * c[3] * gy * Y[4] + c[4] * gx * X[3] + ci * c[4] * gy * Y[3]),
             2.0 * a[..., 0] + a[..., 1] - a[..., 3] - 2.0 * a[..., 4],
             (v + t0 * rho + 2.0 * t1 * fz + 0.4 * t2 * a[..., 4]) * a[..., 0] + (c12 * p[1] + c13 * p[2]) * c[0]
             - ci * 2.0 * (c[0] * gx * X[1] - ci * c[0] * gy * Y[1]) + dp2[..., 0],
             (v + t0 * rho + t1 * fz + 0.4 * t2 * a[..., 3]) * a[..., 1] + (c12.conj() * p[0] + c23 * p[2]) * c[1]
             - ci * 2.0 * (c[1] * gx * X[0] + ci * c[1] * gy * Y[0] + S15 * (c[1] * gx * X[2] - ci * c[1] * gy * Y[2]))
             + dp2[..., 1],
             (v + t0 * rho + 0.2 * t2 * a[..., 2]) * a[..., 2] +
             (c13.conj() * p[0] + c23.conj() * p[1] + c34 * p[3] + c35 * p[4]) * c[2]
             - ci * 2.0 * (S15 * (c[2] * gx * X[1] + ci * c[2] * gy * Y[1] + c[2] * gx * X[3] - ci * c[2] * gy * Y[3]))
             + dp2[..., 2],
             (v + t0 * rho - t1 * fz + 0.4 * t2 * a[..., 1]) * a[..., 3] + (c34.conj() * p[2] + c45 * p[4]) * c[3]
             - ci * 2.0 * (c[3] * gx * X[4] - ci * c[3] * gy * Y[4] + S15 * (c[3] * gx * X[2] + ci * c[3] * gy * Y[2]))
             + dp2[..., 3],
             (v + t0 * rho - 2.0 * t1 * fz + 0.4 * t2 * a[..., 0]) * a[..., 4] + (c35.conj() * p[2] + c45.conj() * p[3]) * c[4]
             - ci * 2.0 * (c[4] * gx * X[3] + ci * c[4] * gy * Y[3]) + dp2[..., 4]]
    ints = [_integrate(np.real(u), dx, dy) for u in t]
    norm = np_normc(phi, dx, dy)
    en = ints[0] / norm.sum()
    mz = ints[1]
    mu = np.array([ints[k + 2] / (norm[k] + EPS) for k in range(2 * spin + 1)])
    return en, mu, mz


def np_rad(phi, x, y, dx, dy):
    r2 = x[:, None] ** 2 + y[None, :] ** 2
    return np.array([np.sqrt(_integrate(r2 * np.abs(phi[..., m]) ** 2, dx, dy)) for m in range(phi.shape[-1])])


@pytest.mark.parametrize("spin", [1, 2])
@pytest.mark.parametrize("gamma", [(0.5, 0.3), (0.0, 0.0)])
def test_oracle_2d_observables_match_numpy_restatement(spin, gamma):
    tau = (200.0, -5.0, 0.0) if spin == 1 else (300.0, 10.0, -8.0)
    kw = dict(dim=2, spin=spin, nx=12, ny=10, nz=1, dx=0.45, dy=0.5, dz=1.0, dt=1e-3, imag=1,
              tau=tau, gx=gamma[0], gy=gamma[1], gz=0.0, ax=1.0, ay=1.3, az=1.0)
    orc = O.Oracle(**kw)
    x, y, _, _, _, _ = orc.grids()
    rng = np.random.default_rng(9)
    g = np.exp(-(x[:, None] ** 2 + y[None, :] ** 2) / 4.0)
    phi = np.stack([g * (1 + 0.2 * rng.standard_normal(g.shape)) * np.exp(1j * rng.uniform(-1, 1, g.shape))
                    for _ in range(2 * spin + 1)], axis=-1)
    orc.set_state(phi.reshape(12, 10, 1, -1))
    en_o, mu_o, mz_o = orc.energy()
    en_n, mu_n, mz_n = np_energy(phi, x, y, kw)
    assert abs(en_o - en_n) <= 1e-12 * abs(en_n)
    assert np.allclose(mu_o, mu_n, rtol=1e-12, atol=1e-12)
    assert abs(mz_o - mz_n) <= 1e-12 * max(1.0, abs(mz_n))
    assert np.allclose(orc.rad(), np_rad(phi, x, y, kw["dx"], kw["dy"]), rtol=1e-12, atol=0)

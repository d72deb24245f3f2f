"""The C oracle's 3D observables against a literal numpy transcription of
cgpe3d.f90 ENERGY 1224-1511 (spin-1 and spin-2, with the GAMMAZ terms), RAD
and NORMC (Simpson over x, then y, then z), FXYZ and MAT_C."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.test_oracle_numpy_2d import EPS, S15, _mat_c, _spin_matrices
from tests.test_oracle_numpy_energy import np_diff
from tests.test_oracle_numpy_projection import np_simpson


def _d(f, axis, h):
    return np.apply_along_axis(np_diff, axis, f.real, h) + 1j * np.apply_along_axis(np_diff, axis, f.imag, h)


def _integrate3(f, dx, dy, dz):
    nx, ny, nz = f.shape
    t1 = np.array([[np_simpson(f[:, j, k], dx) for j in range(ny)] for k in range(nz)])   # [k][j]
    t2 = np.array([np_simpson(t1[k], dy) for k in range(nz)])
    return np_simpson(t2, dz)


def np_observables3d(phi, x, y, z, kw):
    spin, dx, dy, dz = kw["spin"], kw["dx"], kw["dy"], kw["dz"]
    t0, t1, t2 = kw["tau"]
    gx, gy, gz = kw["gx"], kw["gy"], kw["gz"]
    v = (kw["ax"] ** 2 * x[:, None, None] ** 2 + kw["ay"] ** 2 * y[None, :, None] ** 2 +
         kw["az"] ** 2 * z[None, None, :] ** 2)
    ms = 2 * spin + 1
    sx, sy = _spin_matrices(spin)
    fx = np.real(np.einsum("...i,ij,...j->...", phi.conj(), sx, phi))
    fy = np.real(np.einsum("...i,ij,...j->...", phi.conj(), sy, phi))
    a = np.abs(phi) ** 2
    fz = (a * np.arange(spin, -spin - 1, -1)).sum(-1)
    rho = a.sum(-1)
    X = [_d(phi[..., m], 0, dx) for m in range(ms)]
    Y = [_d(phi[..., m], 1, dy) for m in range(ms)]
    Z = [_d(phi[..., m], 2, dz) for m in range(ms)]
    dp2 = [np.abs(X[m]) ** 2 + np.abs(Y[m]) ** 2 + np.abs(Z[m]) ** 2 for m in range(ms)]
    p = [phi[..., m] for m in range(ms)]
    c = [u.conj() for u in p]
    ci = 1j
    if spin == 1:
        r2 = np.sqrt(2.0)
        t = [v * rho + t0 * rho ** 2 / 2.0 + t1 * (fx ** 2 + fy ** 2 + fz ** 2) / 2.0 + sum(dp2) +
             2.0 * np.sqrt(0.5) * (c[0] * (-ci * gx * X[1] - gy * Y[1]) + c[1] * (-ci * gx * X[2] - gy * Y[2]) +
                                   c[1] * (-ci * gx * X[0] + gy * Y[0]) + c[2] * (-ci * gx * X[1] + gy * Y[1])) +
             2.0 * (c[0] * (-ci * gz * Z[0]) + c[2] * (ci * gz * Z[2])),
             a[..., 0] - a[..., 2],
             v * a[..., 0] + dp2[0] + t0 * rho * a[..., 0] + t1 * (a[..., 0] + a[..., 1] - a[..., 2]) * a[..., 0] +
             t1 * c[2] * p[1] ** 2 * c[0] + r2 * (c[0] * (-ci * gx * X[1] - gy * Y[1] - ci * r2 * gz * Z[0])),
             v * a[..., 1] + dp2[1] + t0 * rho * a[..., 1] + t1 * (a[..., 0] + a[..., 2]) * a[..., 1] +
             2.0 * t1 * p[0] * p[2] * c[1] ** 2 +
             r2 * (c[1] * (-ci * gx * X[2] - gy * Y[2]) + c[1] * (-ci * gx * X[0] + gy * Y[0])),
             v * a[..., 2] + dp2[2] + t0 * rho * a[..., 2] + t1 * (a[..., 1] + a[..., 2] - a[..., 0]) * a[..., 2] +
             t1 * c[0] * p[1] ** 2 * c[2] + r2 * (c[2] * (-ci * gx * X[1] + gy * Y[1] + ci * gz * r2 * Z[2]))]
    else:
        r6 = np.sqrt(6.0)
        c12, c13, c23, c34, c35, c45 = _mat_c(phi, kw["tau"])
        theta = (2.0 * p[0] * p[4] - 2.0 * p[1] * p[3] + p[2] ** 2) / np.sqrt(5.0)
        t = [v * rho + sum(dp2) + t0 * rho ** 2 / 2.0 + t1 * (fx ** 2 + fy ** 2 + fz ** 2) / 2.0 +
             t2 * (theta * theta.conj()) / 2.0
             - ci * c[0] * (2.0 * gx * X[1] - ci * 2.0 * gy * Y[1] + 4.0 * gz * Z[0])
             - ci * c[1] * (gx * (2.0 * X[0] + r6 * X[2]) + ci * gy * (2.0 * Y[0] - r6 * Y[2]) + 2.0 * gz * Z[1])
             - ci * c[2] * (gx * r6 * (X[1] + X[3]) + ci * gy * r6 * (Y[1] - Y[3]))
             - ci * c[3] * (gx * (r6 * X[2] + 2.0 * X[4]) + ci * gy * (r6 * Y[2] - 2.0 * Y[4]) - 2.0 * gz * Z[3])
             - ci * c[4] * (2.0 * gx * X[3] + ci * 2.0 * gy * Y[3] - 4.0 * gz * Z[4]),
             2.0 * a[..., 0] + a[..., 1] - a[..., 3] - 2.0 * a[..., 4],
             (v + t0 * rho + 2.0 * t1 * fz + 0.4 * t2 * a[..., 4]) * a[..., 0] + (c12 * p[1] + c13 * p[2]) * c[0]
             - ci * 2.0 * (c[0] * gx * X[1] - ci * c[0] * gy * Y[1] + 2.0 * c[0] * gz * Z[0]) + dp2[0],
             (v + t0 * rho + t1 * fz + 0.4 * t2 * a[..., 3]) * a[..., 1] + (c12.conj() * p[0] + c23 * p[2]) * c[1]
             - ci * 2.0 * (c[1] * gx * X[0] + ci * c[1] * gy * Y[0] +
                           S15 * (c[1] * gx * X[2] - ci * c[1] * gy * Y[2]) + c[1] * gz * Z[1]) + dp2[1],
             (v + t0 * rho + 0.2 * t2 * a[..., 2]) * a[..., 2] +
             (c13.conj() * p[0] + c23.conj() * p[1] + c34 * p[3] + c35 * p[4]) * c[2]
             - ci * 2.0 * (S15 * (c[2] * gx * X[1] + ci * c[2] * gy * Y[1] + c[2] * gx * X[3] - ci * c[2] * gy * Y[3]))
             + dp2[2],
             (v + t0 * rho - t1 * fz + 0.4 * t2 * a[..., 1]) * a[..., 3] + (c34.conj() * p[2] + c45 * p[4]) * c[3]
             - ci * 2.0 * (c[3] * gx * X[4] - ci * c[3] * gy * Y[4] +
                           S15 * (c[3] * gx * X[2] + ci * c[3] * gy * Y[2]) - c[3] * gz * Z[3]) + dp2[3],
             (v + t0 * rho - 2.0 * t1 * fz + 0.4 * t2 * a[..., 0]) * a[..., 4] +
             (c35.conj() * p[2] + c45.conj() * p[3]) * c[4]
             - ci * 2.0 * (c[4] * gx * X[3] + ci * c[4] * gy * Y[3] - 2.0 * c[4] * gz * Z[4]) + dp2[4]]
    ints = [_integrate3(np.real(u), dx, dy, dz) for u in t]
    norm = np.array([_integrate3(a[..., m], dx, dy, dz) for m in range(ms)])
    r2 = x[:, None, None] ** 2 + y[None, :, None] ** 2 + z[None, None, :] ** 2
    rms = np.array([np.sqrt(_integrate3(r2 * a[..., m], dx, dy, dz)) for m in range(ms)])
    en = ints[0] / norm.sum()
    mu = np.array([ints[m + 2] / (norm[m] + EPS) for m in range(ms)])
    return en, mu, ints[1], rms


@pytest.mark.parametrize("spin", [1, 2])
@pytest.mark.parametrize("gamma", [(0.5, 0.3, 0.4), (0.0, 0.0, 0.0)])
def test_oracle_3d_observables_match_numpy_restatement(spin, gamma):
    tau = (200.0, -5.0, 0.0) if spin == 1 else (300.0, 10.0, -8.0)
    kw = dict(dim=3, spin=spin, nx=12, ny=10, nz=8, dx=0.6, dy=0.65, dz=0.7, dt=1e-3, imag=1,
              tau=tau, gx=gamma[0], gy=gamma[1], gz=gamma[2], ax=1.0, ay=1.3, az=1.7)
    orc = O.Oracle(**kw)
    x, y, z, _, _, _ = orc.grids()
    rng = np.random.default_rng(11)
    g = np.exp(-(x[:, None, None] ** 2 + y[None, :, None] ** 2 + z[None, None, :] ** 2) / 4.0)
    phi = np.stack([g * (1 + 0.2 * rng.standard_normal(g.shape)) * np.exp(1j * rng.uniform(-1, 1, g.shape))
                    for _ in range(2 * spin + 1)], axis=-1)
    orc.set_state(phi)
    en_o, mu_o, mz_o = orc.energy()
    en_n, mu_n, mz_n, rms_n = np_observables3d(phi, x, y, z, kw)
    assert abs(en_o - en_n) <= 1e-12 * abs(en_n)
    assert np.allclose(mu_o, mu_n, rtol=1e-12, atol=1e-12)
    assert abs(mz_o - mz_n) <= 1e-12 * max(1.0, abs(mz_n))
    assert np.allclose(orc.rad(), rms_n, rtol=1e-12, atol=0)

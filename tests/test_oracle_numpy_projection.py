"""The C oracle's imaginary-time step without spin-orbit coupling (the
magnetisation projection) against the numpy restatement, from cgpe2d.f90:
the main loop's projection branch 450-476, NEWTON 1286-1331 and USRFUN
1333-1356 (NTRIAL 1000, TOL_NR 1e-6, SIG starting at (20, 20), 432-433),
NORMC 947-986, NORMT 991-1023 and SIMPSON (simpson.f90:4-22), literally.
Three steps on a 2D grid, spin-1 (closed form) and spin-2 (Newton)."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.test_oracle_numpy_2d import EPS, np_ke, np_se, np_sp


def np_simpson(f, dx):
    """simpson.f90:4-22 with its 1-based indices shifted by one."""
    n = len(f)
    f1 = f[1] + f[n - 5]
    f2 = f[2]
    for i in range(4, n - 5, 2):          # Fortran I = 4, N-6, 2
        f1 += f[i - 1]
        f2 += f[i]
    return dx * (f[0] + 4.0 * f1 + 2.0 * f2 + f[n - 4]) / 3.0 + \
        3.0 * dx * (f[n - 4] + 3.0 * (f[n - 3] + f[n - 2]) + f[n - 1]) / 8.0


def np_normc(phi, dx, dy):
    nx, ny, ms = phi.shape
    out = np.zeros(ms)
    for m in range(ms):
        tmp = np.array([np_simpson(np.abs(phi[:, j, m]) ** 2, dx) for j in range(ny)])
        out[m] = np_simpson(tmp, dy)
    return out


def np_normt(phi, dx, dy):
    ny = phi.shape[1]
    tmp = np.array([np_simpson((np.abs(phi[:, j, :]) ** 2).sum(-1), dx) for j in range(ny)])
    return phi / np.sqrt(np_simpson(tmp, dy))


def np_newton(x, n, mag, dt):
    n1, n2, n3, n4, n5 = n
    x = np.array(x, float)
    p = np.zeros(2)
    for _ in range(1000):
        e1 = np.exp(2.0 * (x[0] + 2.0 * x[1]) * dt) * n1
        e2 = np.exp(2.0 * (x[0] + x[1]) * dt) * n2
        e3 = np.exp(2.0 * x[0] * dt) * n3
        e4 = np.exp(2.0 * (x[0] - x[1]) * dt) * n4
        e5 = np.exp(2.0 * (x[0] - 2.0 * x[1]) * dt) * n5
        fv = np.array([e1 + e2 + e3 + e4 + e5 - 1.0, 2.0 * e1 + e2 - e4 - 2.0 * e5 - mag])
        j11 = (e1 + e2 + e3 + e4 + e5) * 2.0 * dt
        j12 = e1 * 4.0 * dt + e2 * 2.0 * dt + e4 * (-2.0 * dt) + e5 * (-4.0 * dt)
        j21 = (2.0 * e1 + e2 - e4 - 2.0 * e5) * 2.0 * dt
        j22 = 2.0 * e1 * 4.0 * dt + e2 * 2.0 * dt - e4 * (-2.0 * dt) - 2.0 * e5 * (-4.0 * dt)
        p[1] = (fv[1] * j11 - fv[0] * j21) / (j21 * j12 - j11 * j22)
        p[0] = (-fv[0] - j12 * p[1]) / j11
        x += p
        if np.abs(p).max() <= 1e-6:
            break
    assert np.abs(p).max() <= 1e-6
    return x


def np_projection_steps(phi, kw, kx, ky, x, y, mag, nsteps):
    spin, dt = kw["spin"], kw["dt"]
    cdt = -1j * dt
    sig = np.array([20.0, 20.0])
    norm = None
    for _ in range(nsteps):
        f = np.fft.fft2(phi, axes=(0, 1))
        f = np_ke(f, kx, ky, cdt)          # SOC with all GAMMA = 0 is the identity
        phi = np.fft.ifft2(f, axes=(0, 1))
        phi = np_se(phi, kw["tau"], cdt, spin)
        phi = np_sp(phi, x, y, kw["ax"], kw["ay"], kw["tau"], cdt, spin)
        norm = np_normc(phi, kw["dx"], kw["dy"])
        if spin == 1:
            n1, n2, n3 = norm
            s2 = np.sqrt(1.0 - mag ** 2) / (np.sqrt(n2 + np.sqrt(4.0 * (1.0 - mag ** 2) * n1 * n3 + mag ** 2 * n2 ** 2)) + EPS)
            s1 = np.sqrt(1.0 + mag - s2 ** 2 * n2) / (np.sqrt(2.0 * n1) + EPS)
            s3 = np.sqrt(1.0 - mag - s2 ** 2 * n2) / (np.sqrt(2.0 * n3) + EPS)
            sigma = np.array([s1, s2, s3])
        else:
            sig = np_newton(sig, norm, mag, dt)
            sigma = np.exp((sig[0] + np.array([2.0, 1.0, 0.0, -1.0, -2.0]) * sig[1]) * dt)
        phi = np_normt(phi * sigma, kw["dx"], kw["dy"])
    return phi, norm, sig


@pytest.mark.parametrize("spin,mag", [(1, 0.1), (2, 0.1), (2, 0.0)])
def test_oracle_projection_steps_match_numpy_restatement(spin, mag):
    tau = (200.0, -5.0, 0.0) if spin == 1 else (300.0, 10.0, -8.0)
    kw = dict(dim=2, spin=spin, nx=12, ny=10, nz=1, dx=0.45, dy=0.5, dz=1.0, dt=1e-3, imag=1,
              tau=tau, gx=0.0, gy=0.0, gz=0.0, ax=1.0, ay=1.3, az=1.0)
    orc = O.Oracle(**kw)
    orc.set_mag(mag)
    x, y, _, kx, ky, _ = orc.grids()
    rng = np.random.default_rng(3)
    g = np.exp(-(x[:, None] ** 2 + y[None, :] ** 2) / 4.0)
    ms = 2 * spin + 1
    phi = np.stack([g * (1 + 0.2 * rng.standard_normal(g.shape)) * np.exp(1j * rng.uniform(-1, 1, g.shape))
                    for _ in range(ms)], axis=-1)
    phi = np_normt(phi, kw["dx"], kw["dy"])
    orc.set_state(phi.reshape(12, 10, 1, ms))
    norm_o = orc.step(3)
    got = orc.state().reshape(phi.shape)
    want, norm_n, sig_n = np_projection_steps(phi, kw, kx, ky, x, y, mag, 3)
    assert np.abs(got - want).max() / np.abs(want).max() < 1e-12
    assert np.allclose(norm_o, norm_n, rtol=1e-12, atol=0)
    if spin == 2:
        assert np.allclose(orc.sig(), sig_n, rtol=1e-10, atol=1e-12)

"""The C oracle's 3D operators against the numpy restatement, from cgpe3d.f90:
KE 875-899 (with the per-component -2 L GAMMAZ KZ term), SOC 904-1004 (the
2D rotation in (kx, ky) applied across kz), SP 1009-1065 (V with the z term,
752), SE 1637-1741 (the same per-point forms as in 2D).  Operator by operator
for spin-1/2 in real and imaginary time, and whole real-time steps with
numpy's FFT."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.test_oracle_numpy_2d import EPS, _soc_matrix, np_se


def np_ke3(phi, kx, ky, kz, gz, cdt, spin):
    e = kx[:, None, None] ** 2 + ky[None, :, None] ** 2 + kz[None, None, :] ** 2
    out = np.empty_like(phi)
    for m in range(2 * spin + 1):
        L = m - spin
        out[..., m] = np.exp(-1j * cdt * (e - 2.0 * L * gz * kz[None, None, :])) * phi[..., m]
    return out


def np_soc3(phi, kx, ky, gx, gy, cdt, spin):
    gkx = gx * kx[:, None] * np.ones_like(ky)[None, :]
    gky = gy * ky[None, :] * np.ones_like(kx)[:, None]
    alpha = 2.0 * np.sqrt(gkx ** 2 + gky ** 2)
    beta = np.where(alpha <= EPS, 0.0, np.arctan2(gky, gkx))
    a = _soc_matrix(spin, beta)[:, :, None]                 # same rotation for every kz
    y = np.einsum("...ji,...j->...i", a.conj(), phi)
    ks = np.arange(-spin, spin + 1)
    y = np.exp(-1j * cdt * ks * alpha[:, :, None, None]) * y
    return np.einsum("...ij,...j->...i", a, y)


def np_sp3(phi, x, y, z, ax, ay, az, tau, cdt, spin):
    t0, t1, t2 = tau
    v = ax * ax * x[:, None, None] ** 2 + ay * ay * y[None, :, None] ** 2 + az * az * z[None, None, :] ** 2
    a = np.abs(phi) ** 2
    base = v + t0 * a.sum(-1)
    if spin == 1:
        t = [base + t1 * (a[..., 0] + a[..., 1] - a[..., 2]), base + t1 * (a[..., 0] + a[..., 2]),
             base + t1 * (a[..., 2] + a[..., 1] - a[..., 0])]
    else:
        fz = 2.0 * a[..., 0] + a[..., 1] - a[..., 3] - 2.0 * a[..., 4]
        t = [base + 2.0 * t1 * fz + 0.4 * t2 * a[..., 4], base + t1 * fz + 0.4 * t2 * a[..., 3],
             base + 0.2 * t2 * a[..., 2], base - t1 * fz + 0.4 * t2 * a[..., 1],
             base - 2.0 * t1 * fz + 0.4 * t2 * a[..., 0]]
    return phi * np.exp(-1j * cdt * np.stack(t, axis=-1))


def _setup(spin, imag, seed=0):
    tau = (200.0, -5.0, 0.0) if spin == 1 else (300.0, 10.0, -8.0)
    kw = dict(dim=3, spin=spin, nx=8, ny=6, nz=10, dx=0.6, dy=0.65, dz=0.7, dt=1e-3 if imag else 5e-4,
              imag=imag, tau=tau, gx=0.5, gy=0.3, gz=0.4, ax=1.0, ay=1.3, az=1.7)
    orc = O.Oracle(**kw)
    rng = np.random.default_rng(seed)
    x, y, z, kx, ky, kz = orc.grids()
    g = np.exp(-(x[:, None, None] ** 2 + y[None, :, None] ** 2 + z[None, None, :] ** 2) / 4.0)
    phi = np.stack([g * (1 + 0.2 * rng.standard_normal(g.shape)) * np.exp(1j * rng.uniform(-1, 1, g.shape))
                    for _ in range(2 * spin + 1)], axis=-1)
    phi = 0.3 * phi / np.abs(phi).max()
    cdt = -1j * kw["dt"] if imag else kw["dt"] + 0j
    return orc, kw, phi, (x, y, z, kx, ky, kz), cdt


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("spin,imag", [(1, 1), (1, 0), (2, 1), (2, 0)])
@pytest.mark.parametrize("op", ["KE", "SOC", "SE", "SP"])
def test_oracle_3d_operator_matches_numpy_restatement(spin, imag, op):
    orc, kw, phi, (x, y, z, kx, ky, kz), cdt = _setup(spin, imag)
    orc.set_state(phi)
    getattr(orc, op.lower())()
    got = orc.state()
    if op == "KE":
        want = np_ke3(phi, kx, ky, kz, kw["gz"], cdt, spin)
    elif op == "SOC":
        want = np_soc3(phi, kx, ky, kw["gx"], kw["gy"], cdt, spin)
    elif op == "SE":
        want = np_se(phi, kw["tau"], cdt, spin)
    else:
        want = np_sp3(phi, x, y, z, kw["ax"], kw["ay"], kw["az"], kw["tau"], cdt, spin)
    assert _rel(got, want) < 1e-12


@pytest.mark.parametrize("spin", [1, 2])
def test_oracle_3d_real_time_steps_match_numpy_restatement(spin):
    orc, kw, phi, (x, y, z, kx, ky, kz), cdt = _setup(spin, 0, seed=1)
    orc.set_state(phi)
    orc.step(3)
    got = orc.state()
    want = phi
    for _ in range(3):
        f = np.fft.fftn(want, axes=(0, 1, 2))
        f = np_ke3(f, kx, ky, kz, kw["gz"], cdt, spin)
        f = np_soc3(f, kx, ky, kw["gx"], kw["gy"], cdt, spin)
        want = np.fft.ifftn(f, axes=(0, 1, 2))
        want = np_se(want, kw["tau"], cdt, spin)
        want = np_sp3(want, x, y, z, kw["ax"], kw["ay"], kw["az"], kw["tau"], cdt, spin)
    assert _rel(got, want) < 1e-12

"""The C oracle's 1D operators and spin-1 observables against the numpy
restatement, from cgpe1d.f90: KE 826-842, SOC 1504-1523 with the fixed
rotation A of INITIALIZE 624-675, SE 1407-1497 (spin-1 with |OMEGA| >= EPS;
spin-2 with the CDT/2 predictor), SP 847-896, ENERGY 1077-1240 (spin-1),
RAD 1036-1072.  Spin-2 in 1D is also pinned by the reference's golden run;
spin-1 is not, which this test backs."""
import numpy as np
import pytest

from oracle import oracle as O
from tests.test_oracle_numpy_2d import EPS, _hmat, _mat_c, _spin_matrices
from tests.test_oracle_numpy_energy import np_diff
from tests.test_oracle_numpy_projection import np_simpson


def _a1d(spin):
    """The fixed SOC rotation of INITIALIZE, cgpe1d.f90:624-675 (A(row, col))."""
    if spin == 1:
        h = np.sqrt(0.5)
        return np.array([[0.5, -h, 0.5], [-h, 0.0, h], [0.5, h, 0.5]])
    q = np.sqrt(0.375)
    a = np.zeros((5, 5))
    a[0, 0], a[1, 0], a[2, 0], a[3, 0], a[4, 0] = 0.25, -0.5, q, -0.5, 0.25
    a[0, 1], a[1, 1], a[2, 1], a[3, 1], a[4, 1] = -0.5, 0.5, 0.0, -0.5, 0.5
    a[0, 2], a[1, 2], a[2, 2], a[3, 2], a[4, 2] = q, 0.0, -0.5, 0.0, q
    a[0, 3], a[1, 3], a[2, 3], a[3, 3], a[4, 3] = -0.5, -0.5, 0.0, 0.5, 0.5
    a[0, 4], a[1, 4], a[2, 4], a[3, 4], a[4, 4] = 0.25, 0.5, q, 0.5, 0.25
    return a


def np_ke1(phi, kx, cdt):
    return phi * np.exp(-1j * cdt * kx ** 2)[:, None]


def np_soc1(phi, kx, gx, cdt, spin):
    a = _a1d(spin)
    y = phi @ a                                        # A^T phi per point
    js = np.arange(-spin, spin + 1)
    y = np.exp(-1j * cdt * 2.0 * js[None, :] * gx * kx[:, None]) * y
    return y @ a.T                                     # A y per point


def np_se1(phi, tau, cdt, spin):
    if spin == 1:
        p0, p1, p2 = phi[:, 0], phi[:, 1], phi[:, 2]
        a1 = tau[1] * p1 * p2.conj()
        b1 = tau[1] * p1 * p0.conj()
        om = cdt * np.sqrt(np.abs(a1) ** 2 + np.abs(b1) ** 2)
        big = np.abs(om) >= EPS
        oms = np.where(big, om, 1.0)
        delta = np.where(big, (np.cos(oms) - 1) / oms ** 2, -0.5)
        kappa = np.where(big, -1j * np.sin(oms) / oms, -1j)
        t1 = delta * cdt ** 2 * (a1 * a1.conj() * p0 + a1 * b1.conj() * p2) + kappa * cdt * a1 * p1
        t2 = delta * cdt ** 2 * (a1 * a1.conj() + b1 * b1.conj()) * p1 + kappa * cdt * (a1.conj() * p0 + b1.conj() * p2)
        t3 = delta * cdt ** 2 * (a1.conj() * b1 * p0 + b1 * b1.conj() * p2) + kappa * cdt * b1 * p1
        return phi + np.stack([t1, t2, t3], axis=-1)
    c = _mat_c(phi, tau)
    phi1 = phi - (1j * cdt / 2.0) * np.einsum("...ij,...j->...i", _hmat(c), phi)
    c1 = _mat_c(phi1, tau)
    w, vec = np.linalg.eigh(_hmat([(u + v) / 2.0 for u, v in zip(c, c1)]))
    y = np.exp(-1j * cdt * w) * np.einsum("...ji,...j->...i", vec.conj(), phi)
    return np.einsum("...ij,...j->...i", vec, y)


def np_sp1(phi, x, ax, tau, cdt, spin):
    t0, t1, t2 = tau
    a = np.abs(phi) ** 2
    base = ax * ax * x ** 2 + t0 * a.sum(-1)
    if spin == 1:
        t = [base + t1 * (a[:, 0] + a[:, 1] - a[:, 2]), base + t1 * (a[:, 0] + a[:, 2]),
             base + t1 * (a[:, 2] + a[:, 1] - a[:, 0])]
    else:
        fz = 2.0 * a[:, 0] + a[:, 1] - a[:, 3] - 2.0 * a[:, 4]
        t = [base + 2.0 * t1 * fz + 0.4 * t2 * a[:, 4], base + t1 * fz + 0.4 * t2 * a[:, 3],
             base + 0.2 * t2 * a[:, 2], base - t1 * fz + 0.4 * t2 * a[:, 1], base - 2.0 * t1 * fz + 0.4 * t2 * a[:, 0]]
    return phi * np.exp(-1j * cdt * np.stack(t, axis=-1))


def np_energy_spin1(phi, x, kw):
    dx, gx, (t0, t1, _) = kw["dx"], kw["gx"], kw["tau"]
    v = kw["ax"] ** 2 * x ** 2
    sx, sy = _spin_matrices(1)
    fx = np.real(np.einsum("...i,ij,...j->...", phi.conj(), sx, phi))
    fy = np.real(np.einsum("...i,ij,...j->...", phi.conj(), sy, phi))
    a = np.abs(phi) ** 2
    fz = a[:, 0] - a[:, 2]
    rho = a.sum(-1)
    d = np.stack([np_diff(phi[:, k].real, dx) + 1j * np_diff(phi[:, k].imag, dx) for k in range(3)], axis=-1)
    dp = np.abs(d) ** 2
    p, c = [phi[:, k] for k in range(3)], [phi[:, k].conj() for k in range(3)]
    r2, ci = np.sqrt(2.0), 1j
    t = [v * rho + t0 * rho ** 2 / 2.0 + t1 * (fx ** 2 + fy ** 2 + fz ** 2) / 2.0 + dp.sum(-1) +
         r2 * gx * (-ci * c[0] * d[:, 1] - ci * c[2] * d[:, 1] - ci * c[1] * (d[:, 0] + d[:, 2])),
         a[:, 0] - a[:, 2],
         v * a[:, 0] + dp[:, 0] + t0 * rho * a[:, 0] + t1 * (a[:, 0] + a[:, 1] - a[:, 2]) * a[:, 0] +
         t1 * c[2] * p[1] ** 2 * c[0] + r2 * gx * (-ci * c[0] * d[:, 1]),
         v * a[:, 1] + dp[:, 1] + t0 * rho * a[:, 1] + t1 * (a[:, 0] + a[:, 2]) * a[:, 1] +
         2.0 * t1 * p[0] * p[2] * c[1] ** 2 + r2 * gx * (-ci * c[1] * (d[:, 0] + d[:, 2])),
         v * a[:, 2] + dp[:, 2] + t0 * rho * a[:, 2] + t1 * (a[:, 1] + a[:, 2] - a[:, 0]) * a[:, 2] +
         t1 * c[0] * p[1] ** 2 * c[2] + r2 * gx * (-ci * c[2] * d[:, 1])]
    ints = [np_simpson(np.real(u), dx) for u in t]
    norm = np.array([np_simpson(a[:, k], dx) for k in range(3)])
    rms = np.array([np.sqrt(np_simpson(x ** 2 * a[:, k], dx)) for k in range(3)])
    return ints[0] / norm.sum(), np.array([ints[k + 2] / (norm[k] + EPS) for k in range(3)]), ints[1], rms


def _setup(spin, imag, seed=0):
    tau = (200.0, -5.0, 0.0) if spin == 1 else (300.0, 10.0, -8.0)
    kw = dict(dim=1, spin=spin, nx=48, dx=0.3, dt=1e-3 if imag else 5e-4, imag=imag, tau=tau,
              gx=0.5, ax=1.0)
    orc = O.Oracle(**kw)
    x, _, _, kx, _, _ = orc.grids()
    rng = np.random.default_rng(seed)
    g = np.exp(-x ** 2 / 4.0)
    phi = np.stack([g * (1 + 0.2 * rng.standard_normal(g.shape)) * np.exp(1j * rng.uniform(-1, 1, g.shape))
                    for _ in range(2 * spin + 1)], axis=-1)
    phi = 0.3 * phi / np.abs(phi).max()
    cdt = -1j * kw["dt"] if imag else kw["dt"] + 0j
    return orc, kw, phi, x, kx, cdt


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("spin,imag", [(1, 1), (1, 0), (2, 1), (2, 0)])
@pytest.mark.parametrize("op", ["KE", "SOC", "SE", "SP"])
def test_oracle_1d_operator_matches_numpy_restatement(spin, imag, op):
    orc, kw, phi, x, kx, cdt = _setup(spin, imag)
    orc.set_state(phi.reshape(48, 1, 1, -1))
    getattr(orc, op.lower())()
    got = orc.state().reshape(phi.shape)
    if op == "KE":
        want = np_ke1(phi, kx, cdt)
    elif op == "SOC":
        want = np_soc1(phi, kx, kw["gx"], cdt, spin)
    elif op == "SE":
        want = np_se1(phi, kw["tau"], cdt, spin)
    else:
        want = np_sp1(phi, x, kw["ax"], kw["tau"], cdt, spin)
    assert _rel(got, want) < 1e-12


@pytest.mark.parametrize("spin", [1, 2])
def test_oracle_1d_real_time_steps_match_numpy_restatement(spin):
    orc, kw, phi, x, kx, cdt = _setup(spin, 0, seed=1)
    orc.set_state(phi.reshape(48, 1, 1, -1))
    orc.step(3)
    got = orc.state().reshape(phi.shape)
    want = phi
    for _ in range(3):
        f = np.fft.fft(want, axis=0)
        f = np_soc1(np_ke1(f, kx, cdt), kx, kw["gx"], cdt, spin)
        want = np.fft.ifft(f, axis=0)
        want = np_sp1(np_se1(want, kw["tau"], cdt, spin), x, kw["ax"], kw["tau"], cdt, spin)
    assert _rel(got, want) < 1e-12


def test_oracle_1d_spin1_observables_match_numpy_restatement():
    orc, kw, phi, x, kx, cdt = _setup(1, 1, seed=2)
    orc.set_state(phi.reshape(48, 1, 1, -1))
    en_o, mu_o, mz_o = orc.energy()
    en_n, mu_n, mz_n, rms_n = np_energy_spin1(phi, x, kw)
    assert abs(en_o - en_n) <= 1e-12 * abs(en_n)
    assert np.allclose(mu_o, mu_n, rtol=1e-12, atol=1e-12)
    assert abs(mz_o - mz_n) <= 1e-12 * max(1.0, abs(mz_n))
    assert np.allclose(orc.rad(), rms_n, rtol=1e-12, atol=0)

"""The C oracle's 2D operators against a second restatement of the
reference's 2D subroutines, written with numpy from cgpe2d.f90:
KE 812-829, SP 834-886, FXYZ 891-913, MAT_C 919-942, SE 1427-1547,
SOC 1554-1650, and the spin matrices SX/SY/SZ of INITIALIZE 634-655.

The numpy side keeps the reference's literal forms: the atan2 rotation
matrices A(beta) of SOC, the cos/sin expressions of the spin-1 SE, and an
eigen-decomposition (numpy.linalg.eigh in place of ZHEEV) for the spin-2 SE.
Grids k, x and y come from the oracle handle, whose grid set-up is pinned by
the golden-run tests.  This backs the 2D, spin-1 and SOC parts of the oracle,
for which the reference ships no output to pin against.
"""
import numpy as np
import pytest

from oracle import oracle as O

EPS = 1.0e-40          # cgpe2d.f90:38
S15 = np.sqrt(1.5)


def _spin_matrices(spin):
    """SX, SY (Fortran RESHAPE fills columns) and SZ, cgpe2d.f90:634-655."""
    if spin == 1:
        sx = np.sqrt(0.5) * np.array([0, 1, 0, 1, 0, 1, 0, 1, 0], float).reshape(3, 3).T
        sy = (1j / np.sqrt(2.0)) * np.array([0, -1, 0, 1, 0, -1, 0, 1, 0], float).reshape(3, 3).T
        return sx, sy
    sx = np.array([0, 1, 0, 0, 0, 1, 0, S15, 0, 0, 0, S15, 0, S15, 0, 0, 0, S15, 0, 1, 0, 0, 0, 1, 0],
                  float).reshape(5, 5).T
    sy = 1j * np.array([0, 1, 0, 0, 0, -1, 0, S15, 0, 0, 0, -S15, 0, S15, 0, 0, 0, -S15, 0, 1, 0, 0, 0, -1, 0],
                       float).reshape(5, 5).T
    return sx, sy


def np_ke(phi, kx, ky, cdt):
    f = np.exp(-1j * cdt * (kx[:, None] ** 2 + ky[None, :] ** 2))
    return phi * f[:, :, None]


def np_sp(phi, x, y, ax, ay, tau, cdt, spin):
    t0, t1, t2 = tau
    v = ax * ax * x[:, None] ** 2 + ay * ay * y[None, :] ** 2
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


def _mat_c(phi, tau):
    """FXYZ + MAT_C: the six upper couplings of the spin-2 SE matrix."""
    sx, sy = _spin_matrices(2)
    fx = np.real(np.einsum("...i,ij,...j->...", phi.conj(), sx, phi))
    fy = np.real(np.einsum("...i,ij,...j->...", phi.conj(), sy, phi))
    fm = fx - 1j * fy
    t1, t2 = tau[1], tau[2]
    p = phi
    return [t1 * fm - 0.4 * t2 * p[..., 3] * p[..., 4].conj(),
            0.2 * t2 * p[..., 2] * p[..., 4].conj(),
            S15 * t1 * fm - 0.2 * t2 * p[..., 2] * p[..., 3].conj(),
            S15 * t1 * fm - 0.2 * t2 * p[..., 1] * p[..., 2].conj(),
            0.2 * t2 * p[..., 0] * p[..., 2].conj(),
            t1 * fm - 0.4 * t2 * p[..., 0] * p[..., 1].conj()]


def _hmat(c):
    c12, c13, c23, c34, c35, c45 = c
    a = np.zeros(c12.shape + (5, 5), complex)
    for (i, j), v in zip(((0, 1), (0, 2), (1, 2), (2, 3), (2, 4), (3, 4)), (c12, c13, c23, c34, c35, c45)):
        a[..., i, j] = v
        a[..., j, i] = v.conj()
    return a


def np_se(phi, tau, cdt, spin):
    if spin == 1:
        p0, p1, p2 = phi[..., 0], phi[..., 1], phi[..., 2]
        a1 = tau[1] * p1 * p2.conj()
        b1 = tau[1] * p1 * p0.conj()
        om = cdt * np.sqrt(np.abs(a1) ** 2 + np.abs(b1) ** 2)
        big = np.abs(om) > EPS
        oms = np.where(big, om, 1.0)
        delta = np.where(big, (np.cos(oms) - 1) / oms ** 2, -0.5)
        kappa = np.where(big, -1j * np.sin(oms) / oms, -1j)
        t1 = delta * cdt ** 2 * (a1 * a1.conj() * p0 + a1 * b1.conj() * p2) + kappa * cdt * a1 * p1
        t2 = delta * cdt ** 2 * (a1 * a1.conj() + b1 * b1.conj()) * p1 + kappa * cdt * (a1.conj() * p0 + b1.conj() * p2)
        t3 = delta * cdt ** 2 * (a1.conj() * b1 * p0 + b1 * b1.conj() * p2) + kappa * cdt * b1 * p1
        return phi + np.stack([t1, t2, t3], axis=-1)
    c = _mat_c(phi, tau)
    phi1 = phi - 1j * cdt * np.einsum("...ij,...j->...i", _hmat(c), phi)
    c1 = _mat_c(phi1, tau)
    h = _hmat([(u + v) / 2.0 for u, v in zip(c, c1)])
    w, vec = np.linalg.eigh(h)
    y = np.einsum("...ji,...j->...i", vec.conj(), phi)
    y = np.exp(-1j * cdt * w) * y
    return np.einsum("...ij,...j->...i", vec, y)


def _soc_matrix(spin, beta):
    e1, e2 = np.exp(-1j * beta), np.exp(-2j * beta)
    if spin == 1:
        a = np.zeros(beta.shape + (3, 3), complex)
        a[..., 0, 0] = 0.5 * e2
        a[..., 1, 0] = -np.sqrt(0.5) * e1
        a[..., 2, 0] = 0.5
        a[..., 0, 1] = -np.sqrt(0.5) * e2
        a[..., 1, 1] = 0.0
        a[..., 2, 1] = np.sqrt(0.5)
        a[..., 0, 2] = a[..., 0, 0]
        a[..., 1, 2] = -a[..., 1, 0]
        a[..., 2, 2] = a[..., 2, 0]
        return a
    a = np.zeros(beta.shape + (5, 5), complex)
    q = np.sqrt(0.375)
    a[..., 0, 0] = 0.25 * e2; a[..., 1, 0] = -0.5 * e1; a[..., 2, 0] = q
    a[..., 3, 0] = a[..., 1, 0].conj(); a[..., 4, 0] = a[..., 0, 0].conj()
    a[..., 0, 1] = -0.5 * e2; a[..., 1, 1] = 0.5 * e1; a[..., 2, 1] = 0.0
    a[..., 3, 1] = -a[..., 1, 1].conj(); a[..., 4, 1] = -a[..., 0, 1].conj()
    a[..., 0, 2] = q * e2; a[..., 1, 2] = 0.0; a[..., 2, 2] = -0.5
    a[..., 3, 2] = 0.0; a[..., 4, 2] = a[..., 0, 2].conj()
    a[..., 0, 3] = -0.5 * e2; a[..., 1, 3] = -0.5 * e1; a[..., 2, 3] = 0.0
    a[..., 3, 3] = -a[..., 1, 3].conj(); a[..., 4, 3] = -a[..., 0, 3].conj()
    a[..., 0, 4] = 0.25 * e2; a[..., 1, 4] = 0.5 * e1; a[..., 2, 4] = q
    a[..., 3, 4] = a[..., 1, 4].conj(); a[..., 4, 4] = a[..., 0, 4].conj()
    return a


def np_soc(phi, kx, ky, gx, gy, cdt, spin):
    gkx = gx * kx[:, None] * np.ones_like(ky)[None, :]
    gky = gy * ky[None, :] * np.ones_like(kx)[:, None]
    alpha = 2.0 * np.sqrt(gkx ** 2 + gky ** 2)
    beta = np.where(alpha <= EPS, 0.0, np.arctan2(gky, gkx))
    a = _soc_matrix(spin, beta)
    y = np.einsum("...ji,...j->...i", a.conj(), phi)
    ks = np.arange(-spin, spin + 1)
    y = np.exp(-1j * cdt * ks[None, None, :] * alpha[..., None]) * y
    return np.einsum("...ij,...j->...i", a, y)


CASES = [(1, 1), (1, 0), (2, 1), (2, 0)]          # spin, imaginary time


def _setup(spin, imag, seed=0):
    nx, ny = 12, 10
    tau = (200.0, -5.0, 0.0) if spin == 1 else (300.0, 10.0, -8.0)
    kw = dict(dim=2, spin=spin, nx=nx, ny=ny, nz=1, dx=0.45, dy=0.5, dz=1.0, dt=1e-3 if imag else 5e-4,
              imag=imag, tau=tau, gx=0.5, gy=0.3, gz=0.0, ax=1.0, ay=1.3, az=1.0)
    orc = O.Oracle(**kw)
    ms = 2 * spin + 1
    rng = np.random.default_rng(seed)
    x, y, _, kx, ky, _ = orc.grids()
    g = np.exp(-(x[:, None] ** 2 + y[None, :] ** 2) / 4.0)
    phi = np.stack([g * (1 + 0.2 * rng.standard_normal(g.shape)) * np.exp(1j * rng.uniform(-1, 1, g.shape))
                    for _ in range(ms)], axis=-1)
    phi = 0.3 * phi / np.abs(phi).max()
    cdt = -1j * kw["dt"] if imag else kw["dt"] + 0j
    return orc, kw, phi, (x, y, kx, ky), cdt


def _rel(a, b):
    return np.abs(a - b).max() / np.abs(b).max()


@pytest.mark.parametrize("spin,imag", CASES)
@pytest.mark.parametrize("op", ["KE", "SOC", "SE", "SP"])
def test_oracle_operator_matches_numpy_restatement(spin, imag, op):
    orc, kw, phi, (x, y, kx, ky), cdt = _setup(spin, imag)
    orc.set_state(phi.reshape(phi.shape[0], phi.shape[1], 1, -1))
    getattr(orc, op.lower())()
    got = orc.state().reshape(phi.shape)
    tau = kw["tau"]
    if op == "KE":
        want = np_ke(phi, kx, ky, cdt)
    elif op == "SOC":
        want = np_soc(phi, kx, ky, kw["gx"], kw["gy"], cdt, spin)
    elif op == "SE":
        want = np_se(phi, tau, cdt, spin)
    else:
        want = np_sp(phi, x, y, kw["ax"], kw["ay"], tau, cdt, spin)
    assert _rel(got, want) < 1e-12


@pytest.mark.parametrize("spin", [1, 2])
def test_oracle_real_time_steps_match_numpy_restatement(spin):
    """Whole real-time split steps (FFT, KE, SOC, BFT, SE, SP; no NORMT in real
    time), with numpy's FFT in place of FFTW."""
    orc, kw, phi, (x, y, kx, ky), cdt = _setup(spin, 0, seed=1)
    orc.set_state(phi.reshape(phi.shape[0], phi.shape[1], 1, -1))
    orc.step(3)
    got = orc.state().reshape(phi.shape)
    want = phi
    for _ in range(3):
        f = np.fft.fft2(want, axes=(0, 1))
        f = np_ke(f, kx, ky, cdt)
        f = np_soc(f, kx, ky, kw["gx"], kw["gy"], cdt, spin)
        want = np.fft.ifft2(f, axes=(0, 1))
        want = np_se(want, kw["tau"], cdt, spin)
        want = np_sp(want, x, y, kw["ax"], kw["ay"], kw["tau"], cdt, spin)
    assert _rel(got, want) < 1e-12

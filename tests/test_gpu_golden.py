"""The GPU path reproduces the reference's only known-answer run (OUTPUT/ of
the 1D spin-2 SO-coupled imaginary-time run of INPUT/input1D.dat) to the
printed precision: file2/file3 rows at 10 decimals, convergence.dat to 1e-9
relative, the exit iteration, the final file1 row and the solution file."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _floats(line):
    return [float(t.replace("D", "E")) for t in line.split()]


@pytest.fixture(scope="module")
def F():
    import fortress_b200 as F
    if not F.device_ok():
        pytest.fail("no usable sm_100 device / libfgpe.so not loaded")
    return F


def _guess(cfg):
    """INITIALIZE's default spin-2 guess, cgpe1d.f90:781-786."""
    x = (-1.0 + 2.0 * np.arange(cfg.n[0]) / cfg.n[0]) * cfg.n[0] * cfg.d[0] / 2.0
    g = np.sqrt(0.2) * np.exp(-cfg.alpha[0] * x * x / 2.0) / np.sqrt(np.sqrt(np.pi))
    return np.repeat(g[:, None], 5, axis=1).astype(np.complex128)


@pytest.fixture(scope="module")
def cfg(F, golden):
    return F.RunConfig.from_text(golden["input1D"], 1)


def test_first_rows(F, cfg, golden):
    from fortress_b200.driver import run
    prop = F.Propagator.from_config(cfg)
    prop.set_state(_guess(cfg))
    res = run(prop, 1600, cfg.stp, cfg.tol, cfg.dt, 1)
    g2, g3, gc = dict(golden["file2"]), dict(golden["file3"]), dict(golden["convergence"])
    for k in range(5):
        assert np.allclose(res.file2[k], _floats(g2[k]), atol=1e-10, rtol=0), k
        assert np.allclose(res.file3[k], _floats(g3[k]), atol=1e-10, rtol=0), k
    for k in range(4):
        g = _floats(gc[k])
        assert abs(res.conv[k][1] - g[1]) <= 1e-9 * g[1]
        assert abs(res.conv[k][2] - g[2]) <= 1e-9 * g[2]


def test_full_run_to_convergence(F, cfg, golden):
    from fortress_b200.driver import run
    prop = F.Propagator.from_config(cfg)
    prop.set_state(_guess(cfg))
    res = run(prop, cfg.niter, cfg.stp, cfg.tol, cfg.dt, 1)
    assert res.final["exited"]
    # "After   399199 iter.:" (the reference reports II-1 on EXIT)
    last = [ln for ln in golden["file1"] if ln.startswith("After ") and "NSTP" not in ln][0]
    assert int(last.split()[1]) == res.final["ii_minus_1"] == 399199
    n_rows = golden["n_rows"]
    assert len(res.conv) == n_rows
    assert len(res.file2) == n_rows       # the exit row is in convergence.dat only
    g2, g3, gc = dict(golden["file2"]), dict(golden["file3"]), dict(golden["convergence"])
    for k, line in g2.items():
        assert np.allclose(res.file2[k], _floats(line), atol=2e-10, rtol=0), k
    for k, line in g3.items():
        assert np.allclose(res.file3[k], _floats(line), atol=2e-10, rtol=0), k
    for k, line in gc.items():
        g = _floats(line)
        assert abs(res.conv[k][0] - g[0]) < 1e-9
        assert abs(res.conv[k][1] - g[1]) <= 1e-7 * g[1], k
    # final file1 row: Norm F7.4, EN and MU F10.5, |phi(center)| F10.5
    vals = _floats(last.split(":")[1])
    assert abs(res.final["norm"].sum() - vals[0]) <= 5e-5
    assert abs(res.final["en"] / 2 - vals[1]) <= 5e-6
    assert np.allclose(res.final["mu"] / 2, vals[2:7], atol=5e-6, rtol=0)
    assert np.allclose(res.final["center"], vals[7:12], atol=5e-6, rtol=0)
    # solution file: x, (density, phase) per component at F18.10
    phi = prop.state().reshape(cfg.n[0], 5)
    rho = np.abs(phi) ** 2
    th = np.arctan2(phi.imag, phi.real)
    for i, line in golden["solution"]:
        v = _floats(line)
        assert np.allclose(rho[i], v[1::2], atol=1e-9, rtol=0), i
        for m in range(5):
            if v[1 + 2 * m] > 1e-6:
                d = abs(th[i, m] - v[2 + 2 * m])
                assert min(d, 2 * np.pi - d) < 1e-6, (i, m)

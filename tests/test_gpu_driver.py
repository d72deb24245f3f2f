"""The drop-in executables (fortress_b200/bin/cgpe{1,2,3}d.x) end to end.

* the reference's own run (INPUT/input1D.dat, 1D spin-2 imaginary time, SOC)
  reproduced file by file against the golden OUTPUT/ to its printed digits;
* 2D/3D runs against the oracle's restatement of the main loop, imaginary
  and real time (the latter started from an initial_sol file)."""
import os
import subprocess

import numpy as np
import pytest

from oracle import oracle as O

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "fortress_b200", "bin")


def _floats(line):
    return [float(t.replace("D", "E")) for t in line.split()]


def _run(tmp, dim, input_text, extra=None, timeout=1800):
    (tmp / "INPUT").mkdir(exist_ok=True)
    (tmp / "OUTPUT").mkdir(exist_ok=True)
    (tmp / "INPUT" / f"input{dim}D.dat").write_text(input_text)
    for name, text in (extra or {}).items():
        (tmp / "INPUT" / name).write_text(text)
    r = subprocess.run([os.path.join(BIN, f"cgpe{dim}d.x")], cwd=tmp, capture_output=True, text=True, timeout=timeout)
    assert r.returncode == 0, r.stderr
    err = (tmp / "err_msg.dat").read_text()
    assert err.strip() == "", err
    return tmp / "OUTPUT"


def test_golden_1d_spin2_full_run(tmp_path, golden):
    out = _run(tmp_path, 1, golden["input1D"])
    f1 = [ln for ln in (out / "file1_im_spin2.dat").read_text().splitlines() if ln.strip()]
    g1 = golden["file1"]
    assert f1[1:12] == g1[1:12]                     # header and table head
    assert len(f1) == len(g1)                       # 39 NSTP rows + final row
    for ours, ref in zip(f1[12:-2], g1[12:-2]):     # table rows and separators
        assert len(ours) == len(ref)
        if not (ref.startswith("Initial") or ref.startswith("After")):
            assert ours == ref
            continue
        assert ours.split(":")[0] == ref.split(":")[0]
        assert np.allclose(_floats(ours.split(":")[1]), _floats(ref.split(":")[1]), atol=1.01e-5, rtol=0), (ours, ref)
    assert f1[-2].startswith("Ended on DAY/MONTH/YEAR") and f1[-1].startswith("Time elapsed = ")
    for name, key in (("file2_im_spin2.dat", "file2"), ("file3_im_spin2.dat", "file3")):
        rows = (out / name).read_text().splitlines()
        assert len(rows) == golden["n_rows"]
        for k, ref in golden[key]:
            assert len(rows[k]) == len(ref)
            assert np.allclose(_floats(rows[k]), _floats(ref), atol=2.01e-10, rtol=0), (k, rows[k], ref)
    conv = (out / "convergence.dat").read_text().splitlines()
    assert len(conv) == golden["n_rows"]
    for k, ref in golden["convergence"]:
        assert len(conv[k]) == len(ref) == 72
        a, b = _floats(conv[k]), _floats(ref)
        assert abs(a[0] - b[0]) < 1e-12
        assert abs(a[1] - b[1]) <= 1e-7 * b[1] and abs(a[2] - b[2]) <= 1e-6 * b[2], (k, conv[k], ref)
    sol = (out / "solution_file_im_spin2.dat").read_text().splitlines()
    assert len(sol) == 2048
    for k, ref in golden["solution"]:
        assert len(sol[k]) == len(ref)
        a, b = _floats(sol[k]), _floats(ref)
        assert abs(a[0] - b[0]) < 1e-9
        assert np.allclose(a[1::2], b[1::2], atol=1.01e-9, rtol=0), (k, sol[k], ref)
        for m in range(5):
            if b[1 + 2 * m] > 1e-6:
                d = abs(a[2 + 2 * m] - b[2 + 2 * m])
                assert min(d, 2 * np.pi - d) < 1e-6


def _input_text(dim, spin, niter, stp, nstp, n, d, dt, a, natoms, nu, tol, im, gamma, fpc=4, mag=0.0):
    lines = [f"{spin}", f"{niter}", f"{stp}, {nstp}", "8", ", ".join(map(str, n)),
             ", ".join(repr(x) for x in list(d) + [dt]), "23", ", ".join(repr(x) for x in a), f"{natoms}",
             ", ".join(map(str, nu)), f"{tol}", f"{im}", ", ".join(repr(g) for g in gamma), f"{fpc}", f"{mag}"]
    return "\n".join(lines) + "\n"


@pytest.mark.parametrize("dim,spin,n,gamma,fpc,mag", [
    (2, 1, (64, 48), (0.6, 0.4), 4, 0.0),
    (2, 2, (48, 48), (0.0, 0.0), 4, 0.25),          # no SOC: Newton projection
    (3, 1, (24, 16, 16), (0.4, 0.3, 0.5), 4, 0.0),
    (1, 1, (256,), (0.0,), 2, 0.3),                 # no SOC, antiferro guess
])
def test_imaginary_time_vs_oracle(tmp_path, dim, spin, n, gamma, fpc, mag):
    d = {1: (0.1,), 2: (0.35, 0.35), 3: (0.6, 0.6, 0.6)}[dim]
    a = (34.9, 45.8, 64.5) if spin == 2 else (50.0, 55.01)
    txt = _input_text(dim, spin, 300, 100, 150, n, d, 5e-4, a, 5000, (20, 25, 400), 1e-12, 1, gamma, fpc, mag)
    out = _run(tmp_path, dim, txt)
    inp = O.Input.parse(txt, dim)
    orc = O.Oracle(**O.params_from_input(inp))
    orc.initialize(inp.option_fpc, inp.mag)
    orc.set_mag(inp.mag)
    ref = O.run_loop(orc, 300, 100, inp.tol, inp.dt, 1)
    sid = spin
    f2 = [_floats(x) for x in (out / f"file2_im_spin{sid}.dat").read_text().splitlines()]
    f3 = [_floats(x) for x in (out / f"file3_im_spin{sid}.dat").read_text().splitlines()]
    cv = [_floats(x) for x in (out / "convergence.dat").read_text().splitlines()]
    assert len(f2) == len(ref["file2"]) == 4 and len(cv) == 3
    for k in range(4):
        assert np.allclose(f2[k], ref["file2"][k], atol=1.5e-10, rtol=0)
        assert np.allclose(f3[k], ref["file3"][k], atol=1.5e-10, rtol=0)
    for k in range(3):
        assert np.allclose(cv[k], ref["conv"][k], rtol=1e-8, atol=0)
    f1 = (out / f"file1_im_spin{sid}.dat").read_text()
    assert "After      300 iter.:" in f1 and f1.count("After NSTP iter.") == 2
    if dim == 3:
        assert (out / f"tmp_solution_file_spin{sid}_xy.dat").exists()


def test_real_time_from_initial_solution(tmp_path):
    """2D spin-2 real time started from an initial_sol file in the solution
    file's own format (x, y, density, phase; blank record after each x)."""
    dim, spin, n = 2, 2, (32, 40)
    gamma = (1.2, 1.0)
    txt = _input_text(dim, spin, 200, 50, 100, n, (0.4, 0.4), 2e-4, (87.93, 91.28, 99.18), 20000,
                      (20, 20, 500), 1e-6, 0, gamma)
    inp = O.Input.parse(txt, dim)
    orc = O.Oracle(**O.params_from_input(inp))
    orc.initialize(4, 0.0)
    rng = np.random.default_rng(2)
    phi = orc.state() * np.exp(1j * rng.uniform(-1, 1, orc.state().shape))
    x, y = orc.grids()[0], orc.grids()[1]
    rows = []
    for i in range(n[0]):
        for j in range(n[1]):
            vals = []
            for m in range(5):
                p = phi[i, j, 0, m]
                vals += [f"{abs(p) ** 2:.17g}", f"{np.arctan2(p.imag, p.real):.17g}"]
            rows.append(f"{x[i]:.17g} {y[j]:.17g} " + " ".join(vals))
        rows.append("")
    out = _run(tmp_path, dim, txt, {"initial_sol_spin2.dat": "\n".join(rows) + "\n"})
    # the oracle starts from the same numbers as read back
    phi2 = np.zeros_like(phi)
    it = iter([r for r in rows if r])
    for i in range(n[0]):
        for j in range(n[1]):
            v = [float(t) for t in next(it).split()]
            for m in range(5):
                phi2[i, j, 0, m] = np.sqrt(v[2 + 2 * m]) * np.exp(1j * v[3 + 2 * m])
    orc.set_state(phi2)
    ref = O.run_loop(orc, 200, 50, inp.tol, inp.dt, 0)
    f2 = [_floats(x) for x in (out / "file2_re_spin2.dat").read_text().splitlines()]
    f3 = [_floats(x) for x in (out / "file3_re_spin2.dat").read_text().splitlines()]
    assert len(f2) == 5 and not (out / "convergence.dat").exists()
    for k in range(5):
        assert np.allclose(f2[k], ref["file2"][k], atol=1.5e-10, rtol=0)
        assert np.allclose(f3[k], ref["file3"][k], atol=1.5e-10, rtol=0)
    sol = [ln for ln in (out / "solution_file_re_spin2.dat").read_text().splitlines()]
    assert len(sol) == n[0] * (n[1] + 1) and sol[n[1]] == ""

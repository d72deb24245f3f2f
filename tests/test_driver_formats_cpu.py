"""Byte layout of the drop-in driver's 2D and 3D output files, on the CPU.

The driver (fortress_b200/driver/cgpe_main.cpp) is built against a host-only
stand-in of libfgpe.so (tests/fake_fgpe/fake_fgpe.c) whose NORMC, ENERGY,
RAD, CONV and state values are deterministic functions of the step count.
The expected files are produced here by a separate Python restatement of the
reference's WRITE statements and their edit descriptors:

* file1 header: cgpe2d.f90:323-370 (formats 899-912), cgpe3d.f90:334-379;
* file1 table: initial row cgpe2d.f90:409-429 (1001-1013), cgpe3d.f90:426-447;
  NSTP rows 1005 and the final row 1006, cgpe2d.f90:521, 548-556,
  cgpe3d.f90:532, 581-583;
* file2/file3 rows '(F14.6,6F18.10)' / '(F14.6,7F18.10)', cgpe2d.f90:436-437,
  513-514; convergence.dat list-directed, cgpe2d.f90:494;
* 2D solution and tmp files '(2F8.2,10F10.5)' with a blank record after
  each x, cgpe2d.f90:522-528 and 562-566;
* 3D solution and tmp files '(10F16.10)', cgpe3d.f90:533-541, 597-603, and
  the xy/xz slices '(2F10.4,10F14.8)', cgpe3d.f90:543-563.
Each line is compared byte for byte (the date and the elapsed time, which
depend on the clock, by pattern).
"""
import math
import os
import re
import shutil
import subprocess

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PI = 4.0 * math.atan(1.0)
AMU, HBAR, AU = 1.66e-27, 1.054560653e-34, 0.529177208e-10


# --------------------------------------------------- Fortran edit descriptors
def F(x, w, d):
    """Fw.d: the optional leading zero goes first when the field is full."""
    s = f"{x:.{d}f}"
    if len(s) > w and s.startswith("0."):
        s = s[1:]
    if len(s) > w and s.startswith("-0."):
        s = "-" + s[2:]
    return "*" * w if len(s) > w else s.rjust(w)


def I(v, w):
    s = str(int(v))
    return "*" * w if len(s) > w else s.rjust(w)


def E(x, w, d):
    """Ew.d: 0.ddddE+ee."""
    if x == 0.0:
        s = "0." + "0" * d + "E+00"
    else:
        e = math.floor(math.log10(abs(x))) + 1
        m = f"{abs(x) / 10.0 ** e:.{d}f}"
        if m.startswith("1"):
            e += 1
            m = f"{abs(x) / 10.0 ** e:.{d}f}"
        s = ("-" if x < 0 else "") + m + f"E{'-' if e < 0 else '+'}{abs(e):02d}"
    return "*" * w if len(s) > w else s.rjust(w)


def ES(x, w, d):
    """ESw.d: d.ddE+ee."""
    m, e = f"{x:.{d}E}".split("E")
    s = f"{m}E{e[0]}{int(e[1:]):02d}"
    return "*" * w if len(s) > w else s.rjust(w)


def LIST(x):
    """One REAL(8) item of list-directed output in the reference's (ifort)
    style, as its shipped convergence.dat shows: F form with 15 significant
    digits and 5 trailing blanks for 0.1 <= |x| < 1e15, else d.dddE-eee, in
    24 columns."""
    a = abs(x)
    if 0.1 <= a < 1e15:
        k = math.floor(math.log10(a)) + 1
        s = f"{x:.{15 - k}f}"
        if len(s) > 17 + (x < 0):
            s = f"{x:.{15 - k - 1}f}"
        return s.rjust(19) + "     "
    if x == 0.0:
        return "  0.000000000000000E+000"
    e = math.floor(math.log10(a))
    m = f"{a / 10.0 ** e:.15f}"
    if m.startswith("10"):
        e += 1
        m = f"{a / 10.0 ** e:.15f}"
    return (("-" if x < 0 else "") + m + f"E{'-' if e < 0 else '+'}{abs(e):03d}").rjust(24)


# ------------------------------------------------------ the fake library's values
def fake_norm(ms, c):
    return [0.1 + 0.05 * m + 1e-7 * c for m in range(ms)]


def fake_obs(ms, c):
    en = 3.0 + 1.0 / (1.0 + c)
    return en, [en + 0.1 * m for m in range(ms)], 1e-5 * c, [1.5 + 0.01 * m + 1e-6 * c for m in range(ms)]


def fake_dphi(c):
    return 1e-3 / (1.0 + c)


# -------------------------------------------------------------------- builds
@pytest.fixture(scope="module")
def drivers(tmp_path_factory):
    if not shutil.which("gcc") or not shutil.which("g++"):
        pytest.skip("needs gcc/g++")
    d = tmp_path_factory.mktemp("fakelib")
    subprocess.run(["gcc", "-O1", "-shared", "-fPIC", "-o", str(d / "libfgpe.so"),
                    os.path.join(ROOT, "tests", "fake_fgpe", "fake_fgpe.c")], check=True)
    exe = {}
    for dim in (2, 3):
        out = d / f"cgpe{dim}d.x"
        subprocess.run(["g++", "-O1", "-std=c++17", f"-DFGPE_DIMENSION={dim}", "-o", str(out),
                        os.path.join(ROOT, "fortress_b200", "driver", "cgpe_main.cpp"), f"-L{d}", "-lfgpe",
                        f"-Wl,-rpath,{d}"], check=True)
        exe[dim] = str(out)
    return exe


# --------------------------------------------------------------------- cases
def input_text(case):
    dim, spin = case["dim"], case["spin"]
    L = [f"{spin}", f"{case['niter']}", f"{case['stp']} {case['nstp']}", "8",
         " ".join(str(v) for v in case["n"][:dim]),
         " ".join(repr(v) for v in case["d"][:dim]) + f" {case['dt']!r}",
         f"{case['mass']!r}", " ".join(repr(v) for v in case["a"][: (2 if spin == 1 else 3)]),
         f"{case['natoms']}", " ".join(repr(v) for v in case["nu"]), f"{case['tol']!r}",
         f"{case['im']}", " ".join(repr(v) for v in case["gamma"][:dim]), "4", "0.0"]
    return "\n".join(L) + "\n"


def derived(case):
    dim, spin = case["dim"], case["spin"]
    nux, nuy, nuz = case["nu"]
    al = (nux / nux, nuy / nux, nuz / nux)
    aosc = math.sqrt(HBAR / (case["mass"] * AMU * 2.0 * PI * nux))
    geo = math.sqrt(al[2] / (2.0 * PI)) if dim == 2 else 1.0
    A0, A2, A4 = (list(case["a"]) + [0.0])[:3]
    if spin == 1:
        na = float(np.float32(case["natoms"]))          # REAL(NATOMS)
        tau = [2.0 * geo * (4.0 * PI * na * (A0 * AU + 2.0 * A2 * AU) / (3.0 * aosc)),
               2.0 * geo * (4.0 * PI * na * (A2 * AU - A0 * AU) / (3.0 * aosc)), 0.0]
    else:
        nd = float(case["natoms"])
        tau = [2.0 * (geo * 4.0 * PI * nd * (4.0 * A2 * AU + 3.0 * A4 * AU) / (7.0 * aosc)),
               2.0 * (geo * 4.0 * PI * nd * (A4 * AU - A2 * AU) / (7.0 * aosc)),
               2.0 * (geo * 4.0 * PI * nd * (7.0 * A0 * AU - 10.0 * A2 * AU + 3.0 * A4 * AU) / (7.0 * aosc))]
    return al, aosc, tau


def grid(case, a):
    n, d = case["n"][a], case["d"][a]
    return [(-1.0 + 2.0 * (i - 1.0) / n) * n * d / 2.0 for i in range(1, n + 1)]


def state_and_file(case, rng):
    """Real time: the initial_sol file text (coordinates shifted off the
    grid so the read-back X/Y show in the outputs) and the state the driver
    builds from it; imaginary time: INITIALIZE's default guess."""
    dim, spin = case["dim"], case["spin"]
    ms = 2 * spin + 1
    n = [case["n"][a] if a < dim else 1 for a in range(3)]
    X = [grid(case, a) if a < dim else [0.0] for a in range(3)]
    if case["im"]:
        al, _, _ = derived(case)
        x2 = np.asarray(X[0])[:, None, None] ** 2
        y2 = np.asarray(X[1])[None, :, None] ** 2
        z2 = np.asarray(X[2])[None, None, :] ** 2
        if dim == 2:
            g = np.exp(-(al[0] * x2 + al[1] * y2) / 2.0) / math.sqrt(PI)
        else:
            g = np.exp(-(al[0] * x2 + al[1] * y2 + al[2] * z2) / 2.0) / PI ** 0.75
        if spin == 1:
            gg = np.exp(-(x2 + y2 + z2) / 2.0) / PI ** 0.75 if dim == 3 else g
            comps = [gg] * 3
        else:
            comps = [(1.0 if dim == 3 else math.sqrt(0.2)) * g] * 5
        return None, np.stack(comps, axis=-1).astype(complex), X
    rho = rng.uniform(0.001, 0.9, size=tuple(n) + (ms,))
    th = rng.uniform(-3.0, 3.0, size=tuple(n) + (ms,))
    Xr = [list(X[0]), list(X[1]), list(X[2])]
    lines = []
    for i in range(n[0]):
        for j in range(n[1]):
            for k in range(n[2]):
                vals = []
                if dim == 2:
                    xi, yj = X[0][i] + 0.001 * (i + 1), X[1][j] - 0.002 * (j + 1)
                    Xr[0][i], Xr[1][j] = xi, yj
                    vals = [f"{xi:.17g}", f"{yj:.17g}"]
                for m in range(ms):
                    vals += [f"{rho[i, j, k, m]:.17g}", f"{th[i, j, k, m]:.17g}"]
                lines.append(" ".join(vals))
    phi = np.sqrt(rho) * np.exp(1j * th)
    return "\n".join(lines) + "\n", phi, Xr


def expected(case, phi, X, XR):
    """Every output file of the run, as the reference's WRITE statements
    lay them out for the fake library's values."""
    dim, spin = case["dim"], case["spin"]
    ms = 2 * spin + 1
    im = case["im"]
    al, aosc, tau = derived(case)
    n = [case["n"][a] if a < dim else 1 for a in range(3)]
    niter, stp, nstp, dt, tol = case["niter"], case["stp"], case["nstp"], case["dt"], case["tol"]
    g, dd = case["gamma"], case["d"]
    c2 = [n[0] // 2, n[1] // 2, n[2] // 2]
    center = [abs(phi[c2[0], c2[1], c2[2], m]) for m in range(ms)]
    f1 = [None, " "]                                                # date (1007), WRITE(2,*)
    f1.append(" OPENMP_THREADS = " + I(8, 3) + ", FFTW_THREADS = " + I(8, 3))
    gam = ", GAMMAX = " + F(g[0], 6, 2) + ", GAMMAY = " + F(g[1], 6, 2)
    if dim == 3:
        gam += ", GAMMAZ = " + F(g[2], 6, 2)
    f1.append(" SWITCH_IM = " + I(im, 2) + ", OPTION_FPC = " + I(4, 2) + ", SWITCH_SOC = " + I(1, 2) + gam +
              ", TOL = " + ES(tol, 9, 2))
    f1.append(" Anisotropy ALPHAX =" + F(al[0], 12, 6) + ", ALPHAY = " + F(al[1], 12, 6) + ", ALPHAZ = " +
              F(al[2], 12, 6))
    f1.append(" ")
    if dim == 2:
        f1.append(" No. of space steps NX = " + I(n[0], 8) + ", NY = " + I(n[1], 8))
        f1.append(" No. of time steps : NITER = " + I(niter, 9) + ", NSTP = " + I(nstp, 9) + ", STP = " + I(stp, 9))
        f1.append(" Space Step DX = " + F(dd[0], 10, 6) + ", DY = " + F(dd[1], 10, 6))
        f1.append(" Time Step  DT = " + F(dt, 10, 6) + ", MAG = " + F(0.0, 12, 6))
    else:
        f1.append(" No. of space steps NX = " + I(n[0], 8) + ", NY = " + I(n[1], 8) + ", NZ = " + I(n[2], 8))
        f1.append(" No. of time steps : NITER = " + I(niter, 9) + ", NSTP = " + I(nstp, 9) + ", STP = " + I(stp, 9))
        f1.append(" Spatial step-size DX = " + F(dd[0], 10, 6) + ", DY = " + F(dd[1], 10, 6) + ", DZ = " +
                  F(dd[2], 10, 6))
        f1.append(" Temporal step-size  DT = " + F(dt, 10, 6) + ", MAG = " + F(0.0, 12, 6))
    f1.append(" ")
    f1.append(" AOSC = " + E(aosc, 12, 4))
    a = case["a"]
    if spin == 1 and dim == 2:
        f1.append(" A0 = " + F(a[0], 12, 6) + ", A2 = " + F(a[1], 12, 6) + ",  (all in units of Bohr radius) ")
        f1.append(" TAU(0) = " + F(tau[0] / 2, 12, 6) + ", TAU(1) = " + F(tau[1] / 2, 12, 6) +
                  " (in dimensionless units)")
    elif spin == 1:
        f1.append(" A0 = " + F(a[0], 12, 6) + ", A2 = " + F(a[1], 12, 6) + " (all in units of Bohr radius)")
        f1.append(" TAU(0) = " + F(tau[0] / 2, 12, 6) + ", TAU(1) = " + F(tau[1] / 2, 12, 6) +
                  " in dimensionless units ")
    else:
        f1.append(" A0 = " + F(a[0], 12, 6) + ", A2 = " + F(a[1], 12, 6) + ", A4 = " + F(a[2], 12, 6) +
                  " (all in units of Bohr radius) ")
        f1.append(" TAU(0) = " + F(tau[0] / 2, 12, 6) + ", TAU(1) = " + F(tau[1] / 2, 12, 6) + ", TAU(2) = " +
                  F(tau[2] / 2, 12, 6) + " (in dimensionless units)")
    f1.append(" ")
    if spin == 1:
        sep = " " * 23 + "-" * (74 if dim == 3 else 76)
        hdr = " " * 23 + "Norm" + " " * 7 + "EN" + " " * 7 + "MU1" + " " * 7 + "MU2" + " " * 7 + "MU3" + " " * 6 + \
            "phi1" + " " * 6 + "phi2" + " " * 6 + "phi3"
        lead0 = "Initial: " + " " * 8
    else:
        sep = " " * 22 + "-" * 117
        hdr = " " * 23 + "Norm" + " " * 7 + "EN" + "".join(" " * 7 + f"MU{k}" for k in range(1, 6)) + " " * 7 + \
            "phi1" + " " * 7 + "phi2" + " " * 5 + "phi3" + " " * 5 + "phi4" + " " * (6 if dim == 3 else 5) + "phi5"
        lead0 = "Initial : " + " " * 7
    f1 += [sep, hdr, sep]
    norm = fake_norm(ms, 0)
    en, mu, mz, rms = fake_obs(ms, 0)
    f1.append(lead0 + F(sum(norm), 11, 4) + F(en / 2, 10, 5) + "".join(F(v / 2, 10, 5) for v in mu) +
              "".join(F(v, 10, 5) for v in center))

    def r2(t, en, rms):
        return F(t, 14, 6) + F(en / 2, 18, 10) + "".join(F(v, 18, 10) for v in rms)

    def r3(t, norm, mz):
        return F(t, 14, 6) + "".join(F(v, 18, 10) for v in norm) + F(sum(norm), 18, 10) + F(mz, 18, 10)

    f2, f3, conv = [r2(0.0, en, rms)], [r3(0.0, norm, mz)], []
    en_old = en
    nstp_lead = "After NSTP iter.:    " if dim == 3 else "After NSTP iter.    :"
    exited = False
    tmp_written = False
    for ii in range(1, niter + 1):
        norm = fake_norm(ms, ii)
        if ii % stp == 0:
            en, mu, mz, rms = fake_obs(ms, ii)
            if im:
                cv = fake_dphi(ii) / (stp * 2.0 * dt)
                ce = abs(en - en_old) / (stp * 2.0 * dt)
                conv.append(LIST(2.0 * ii * dt) + LIST(cv) + LIST(ce))
                if cv <= tol or ce <= tol:
                    exited = True
                    break
            f2.append(r2(2.0 * ii * dt, en, rms))
            f3.append(r3(2.0 * ii * dt, norm, mz))
        en_old = en
        if ii % nstp == 0:
            f1.append(nstp_lead + F(sum(norm), 7, 4) + F(en / 2, 10, 5) + "".join(F(v / 2, 10, 5) for v in mu) +
                      "".join(F(v, 10, 5) for v in center))
            tmp_written = True
    c_final = ii if exited else niter
    en, mu, mz, rms = fake_obs(ms, c_final)
    f1.append(sep)
    f1.append("After " + I(ii - 1 if exited else niter, 8) + " iter.:" + F(sum(norm), 7, 4) + F(en / 2, 10, 5) +
              "".join(F(v / 2, 10, 5) for v in mu) + "".join(F(v, 10, 5) for v in center))
    f1 += [sep, " ", None, None]                                   # 1008 date, 1009 elapsed
    rho, th = np.abs(phi) ** 2, np.arctan2(phi.imag, phi.real)
    sol, slices = [], {}
    if dim == 2:
        for i in range(n[0]):
            for j in range(n[1]):
                sol.append(F(XR[0][i], 8, 2) + F(XR[1][j], 8, 2) +
                           "".join(F(rho[i, j, 0, m], 10, 5) + F(th[i, j, 0, m], 10, 5) for m in range(ms)))
            sol.append("")
    else:
        for i in range(n[0]):
            for j in range(n[1]):
                for k in range(n[2]):
                    sol.append("".join(F(rho[i, j, k, m], 16, 10) + F(th[i, j, k, m], 16, 10) for m in range(ms)))
        for name, (ax, other) in {"xy": (1, 2), "xz": (2, 1)}.items():
            lines = []
            for i in range(n[0]):
                for b in range(n[ax]):
                    idx = [i, 0, 0]
                    idx[ax] = b
                    idx[other] = n[other] // 2
                    lines.append(F(X[0][i], 10, 4) + F(X[ax][b], 10, 4) +
                                 "".join(F(rho[tuple(idx) + (m,)], 14, 8) + F(th[tuple(idx) + (m,)], 14, 8)
                                         for m in range(ms)))
                lines.append("")
            slices[name] = lines
    return dict(file1=f1, file2=f2, file3=f3, conv=conv if im else None, solution=sol,
                tmp=sol if tmp_written else None, slices=slices if tmp_written else {})


CASES = [
    dict(dim=2, spin=1, im=1, n=(16, 12), d=(0.2, 0.25, 1.0), dt=0.001, niter=80, stp=10, nstp=20, tol=1e-3,
         mass=87.0, a=(101.8, 100.4), natoms=20000, nu=(20.0, 30.0, 400.0), gamma=(0.5, 0.75)),
    dict(dim=2, spin=2, im=0, n=(12, 10), d=(0.3, 0.3, 1.0), dt=0.0001, niter=40, stp=10, nstp=20, tol=1e-8,
         mass=87.0, a=(87.93, 91.28, 99.18), natoms=50000, nu=(20.0, 20.0, 500.0), gamma=(1.2, 1.0)),
    dict(dim=3, spin=1, im=1, n=(8, 6, 10), d=(0.4, 0.5, 0.3), dt=0.001, niter=80, stp=10, nstp=20, tol=1e-3,
         mass=87.0, a=(101.8, 100.4), natoms=100000, nu=(50.0, 50.0, 50.0), gamma=(0.5, 0.5, 0.5)),
    dict(dim=3, spin=2, im=0, n=(6, 8, 4), d=(0.4, 0.4, 0.5), dt=0.0005, niter=30, stp=10, nstp=15, tol=1e-8,
         mass=23.0, a=(34.9, 45.8, 64.5), natoms=10000, nu=(20.0, 25.0, 30.0), gamma=(0.3, 0.2, 0.1)),
]


def _id(c):
    return f"{c['dim']}d-spin{c['spin']}-{'im' if c['im'] else 're'}"


def _lines(path):
    with open(path) as f:
        return f.read().split("\n")[:-1]


def _compare(got, want, what):
    assert len(got) == len(want), f"{what}: {len(got)} lines, expected {len(want)}"
    for k, (g, w) in enumerate(zip(got, want)):
        if w is None:
            continue
        assert g == w, f"{what} line {k + 1}:\n got  {g!r}\n want {w!r}"


@pytest.mark.parametrize("case", CASES, ids=_id)
def test_output_files_match_reference_formats(drivers, tmp_path, case):
    dim, spin, im = case["dim"], case["spin"], case["im"]
    rng = np.random.default_rng(7)
    init_text, phi, XR = state_and_file(case, rng)
    X = [grid(case, a) if a < dim else [0.0] for a in range(3)]
    (tmp_path / "INPUT").mkdir()
    (tmp_path / "OUTPUT").mkdir()
    (tmp_path / "INPUT" / f"input{dim}D.dat").write_text(input_text(case))
    if init_text is not None:
        (tmp_path / "INPUT" / f"initial_sol_spin{spin}.dat").write_text(init_text)
    r = subprocess.run([drivers[dim]], cwd=tmp_path, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0, r.stdout + r.stderr
    want = expected(case, phi, X, XR)
    tag = f"{'im' if im else 're'}_spin{spin}"
    out = tmp_path / "OUTPUT"
    f1 = _lines(out / f"file1_{tag}.dat")
    _compare(f1, want["file1"], "file1")
    date = r"(Started|Ended) on DAY/MONTH/YEAR, HOURS:MINUTES:SECONDS = [ \d]{2}/[ \d]{2}/\d{4},[ \d]{3}:[ \d]{2}:[ \d]{2}"
    assert re.fullmatch(date, f1[0]) and f1[0].startswith("Started")
    assert re.fullmatch(date, f1[-2]) and f1[-2].startswith("Ended")
    assert re.fullmatch(r"Time elapsed = [ \d.]{18} in seconds", f1[-1])
    _compare(_lines(out / f"file2_{tag}.dat"), want["file2"], "file2")
    _compare(_lines(out / f"file3_{tag}.dat"), want["file3"], "file3")
    if want["conv"] is not None:
        _compare(_lines(out / "convergence.dat"), want["conv"], "convergence.dat")
    _compare(_lines(out / f"solution_file_{tag}.dat"), want["solution"], "solution file")
    if want["tmp"] is not None:
        _compare(_lines(out / f"tmp_solution_file_spin{spin}.dat"), want["tmp"], "tmp solution file")
    for name, lines in want["slices"].items():
        _compare(_lines(out / f"tmp_solution_file_spin{spin}_{name}.dat"), lines, f"{name} slice")

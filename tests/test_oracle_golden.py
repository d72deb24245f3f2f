"""Pin the CPU oracle against the reference's only known-answer output
(OUTPUT/ of the 1D spin-2 SO-coupled imaginary-time run of INPUT/input1D.dat).

Printed precision: file2/file3 rows carry 10 decimals (F18.10), the header
TAU/2 values 6 decimals (F12.6), convergence.dat full list-directed precision.
"""
import numpy as np
import pytest

from oracle import oracle as O


def _floats(line):
    return [float(t.replace("D", "E")) for t in line.split()]


@pytest.fixture(scope="module")
def inp(golden):
    return O.Input.parse(golden["input1D"], 1)


def test_input_records(inp):
    assert inp.spin == 2 and inp.n[0] == 2048 and inp.stp == 400 and inp.nstp == 10000
    assert inp.switch_im == 1 and inp.switch_soc == 1 and inp.gamma[0] == 0.5
    assert inp.dt == 0.000125 and inp.d[0] == 0.05


def test_tau_and_aosc_header(inp, golden):
    tau, aosc = inp.tau()
    # " TAU(0) =   242.966174, TAU(1) =    12.061236, TAU(2) =   -13.028714 ..."
    line = [ln for ln in golden["file1"] if ln.startswith(" TAU(0)")][0]
    printed = [float(x.split("=")[1]) for x in line.split("(in")[0].split(",")]
    assert np.allclose(tau / 2.0, printed, atol=5e-7, rtol=0)
    aline = [ln for ln in golden["file1"] if ln.startswith(" AOSC")][0]
    assert abs(aosc - float(aline.split("=")[1])) <= 0.5e-9  # E12.4: 0.4688E-05


@pytest.fixture(scope="module")
def run1600(inp):
    orc = O.Oracle(**O.params_from_input(inp))
    orc.initialize(inp.option_fpc, inp.mag)
    return O.run_loop(orc, 1600, inp.stp, inp.tol, inp.dt, 1)


def test_initial_row(run1600, golden):
    ini = run1600["initial"]
    row = [ln for ln in golden["file1"] if ln.startswith("Initial")][0]
    vals = _floats(row.split(":")[1])
    assert abs(ini["norm"].sum() - vals[0]) < 5e-5
    assert abs(ini["en"] / 2 - vals[1]) < 5e-6
    assert np.allclose(ini["mu"] / 2, vals[2:7], atol=5e-6, rtol=0)


@pytest.mark.parametrize("k", range(5))
def test_file2_file3_rows(run1600, golden, k):
    g2 = dict(golden["file2"])[k]
    g3 = dict(golden["file3"])[k]
    ours2 = run1600["file2"][k]
    ours3 = run1600["file3"][k]
    assert np.allclose(ours2, _floats(g2), atol=1e-10, rtol=0), (ours2, g2)
    assert np.allclose(ours3, _floats(g3), atol=1e-10, rtol=0), (ours3, g3)


@pytest.mark.parametrize("k", range(4))
def test_convergence_rows(run1600, golden, k):
    g = _floats(dict(golden["convergence"])[k])
    ours = run1600["conv"][k]
    assert abs(ours[0] - g[0]) < 1e-12
    assert abs(ours[1] - g[1]) <= 1e-9 * abs(g[1])
    assert abs(ours[2] - g[2]) <= 1e-9 * abs(g[2])

"""The drop-in executable's input parsing and file1 header (written before
the device is needed) against the reference's golden file1, with no GPU
visible: the program must stop cleanly with a message in err_msg.dat."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "fortress_b200", "bin")


@pytest.fixture(scope="module")
def exe():
    path = os.path.join(BIN, "cgpe1d.x")
    if not os.path.exists(path):
        pytest.skip("driver not built (fortress_b200.build.build())")
    return path


def test_header_matches_golden_without_gpu(tmp_path, exe, golden):
    (tmp_path / "INPUT").mkdir()
    (tmp_path / "OUTPUT").mkdir()
    (tmp_path / "INPUT" / "input1D.dat").write_text(golden["input1D"])
    env = dict(os.environ, CUDA_VISIBLE_DEVICES="")
    r = subprocess.run([exe], cwd=tmp_path, env=env, capture_output=True, text=True, timeout=120)
    assert r.returncode == 0                      # Fortran STOP semantics
    ours = [ln for ln in (tmp_path / "OUTPUT" / "file1_im_spin2.dat").read_text().splitlines() if ln.strip()]
    gold = golden["file1"]
    # line 0 is the start date; 1..10 the parameter block (blank lines dropped)
    assert ours[0].startswith("Started on DAY/MONTH/YEAR, HOURS:MINUTES:SECONDS = ")
    assert len(ours[0]) == len(gold[0])
    assert ours[1:11] == gold[1:11]
    err = (tmp_path / "err_msg.dat").read_text()
    assert "fgpe error" in err


def test_missing_input(tmp_path, exe):
    r = subprocess.run([exe], cwd=tmp_path, capture_output=True, text=True, timeout=60)
    assert r.returncode == 0
    assert "'input1D.dat' does not exist." in (tmp_path / "err_msg.dat").read_text()

"""The C-ABI library on a machine without a GPU: it loads, exports every
function include/fgpe.h declares, its parameter structure matches the C
layout, and every entry point that needs the device fails loudly (no CPU
fallback)."""
import ctypes
import os
import re
import subprocess

import pytest

from fortress_b200 import _abi

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def _declared():
    text = open(os.path.join(ROOT, "include", "fgpe.h")).read()
    return sorted(set(re.findall(r"\b(fgpe_[a-z0-9_]+)\s*\(", text)))


def test_header_symbols_exported():
    lib = _abi.load()
    declared = _declared()
    assert len(declared) >= 30
    for name in declared:
        assert hasattr(lib, name), name
    assert set(declared) == set(_abi.EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (fgpe_[a-z0-9_]+)", out))
    assert exported == set(declared)


def test_fno_header_symbols_exported():
    from fortress_b200 import fno
    hdr = open(os.path.join(ROOT, "include", "fno.h")).read()
    declared = set(re.findall(r"^int (fno_[a-z0-9_]+)\(", hdr, re.M))
    assert declared == set(fno.FNO_EXPORTS)
    out = subprocess.run(["nm", "-D", "--defined-only", _abi.LIB_PATH], capture_output=True, text=True).stdout
    assert set(re.findall(r" T (fno_[a-z0-9_]+)", out)) == declared
    L = fno.lib()                      # argtypes bind without a device
    assert L.fno_gemm.restype is not None


def test_params_layout_matches_c(tmp_path):
    src = tmp_path / "layout.c"
    src.write_text('#include <stdio.h>\n#include <stddef.h>\n#include "fgpe.h"\n'
                   'int main(){printf("%zu %zu %zu %zu",sizeof(fgpe_params),offsetof(fgpe_params,tau),'
                   'offsetof(fgpe_params,kernels),offsetof(fgpe_params,mag));}\n')
    env = dict(os.environ)
    env.pop("CC", None)
    subprocess.run(["gcc", "-I", os.path.join(ROOT, "include"), "-o", str(tmp_path / "layout"), str(src)], check=True, env=env)
    got = subprocess.run([str(tmp_path / "layout")], capture_output=True, text=True).stdout.split()
    P = _abi.Params
    assert [int(x) for x in got] == [ctypes.sizeof(P), P.tau.offset, P.kernels.offset, P.mag.offset]


def _no_gpu():
    try:
        import torch
        return not torch.cuda.is_available()
    except Exception:
        return True


@pytest.mark.skipif(not _no_gpu(), reason="checks the behaviour without a device")
def test_fails_loudly_without_device():
    import fortress_b200 as F
    from fortress_b200.batch import Batch
    assert _abi.load().fgpe_device_ok() == 0
    assert not F.device_ok()
    kw = dict(dim=2, spin=1, n=(32, 32), d=(0.1, 0.1), dt=1e-3, imag_time=1, tau=(1.0, 0.0, 0.0))
    with pytest.raises(F.FgpeError) as e:
        F.Propagator(**kw)
    assert e.value.code == _abi.FGPE_E_CUDA
    with pytest.raises(F.FgpeError):
        Batch([kw, kw])


def test_argument_errors_need_no_device():
    import fortress_b200 as F
    with pytest.raises(F.FgpeError) as e:
        F.Propagator(dim=4, spin=1, n=(32,), d=(0.1,), dt=1e-3, imag_time=1, tau=(1.0, 0.0, 0.0))
    assert e.value.code == _abi.FGPE_E_ARG
    with pytest.raises(F.FgpeError):
        F.Propagator(dim=2, spin=1, n=(32, 14), d=(0.1, 0.1), dt=1e-3, imag_time=1, tau=(1.0, 0.0, 0.0))
    with pytest.raises(F.FgpeError):
        F.Propagator(dim=1, spin=1, n=(32,), d=(0.1,), dt=-1.0, imag_time=1, tau=(1.0, 0.0, 0.0))


def test_fno_gemm_tc_argument_errors_need_no_device():
    from fortress_b200 import fno
    L = fno.lib()
    p = ctypes.c_void_p(16)            # never dereferenced: the checks come first
    ok = (2, 8, 8, 8, 1.0, p, 0, 64, 8, 1, p, 0, 8, 1, 0.0, p, 64, 8, 1)
    assert L.fno_gemm_tc(*ok[:5], None, *ok[6:], p, None) == _abi.FGPE_E_ARG       # null A
    assert L.fno_gemm_tc(*ok, None, None) == _abi.FGPE_E_ARG                       # null error flag
    assert L.fno_gemm_tc(0, *ok[1:], p, None) == _abi.FGPE_E_ARG                   # empty batch
    bad = list(ok)
    bad[12] = -1                                                                   # negative sBb
    assert L.fno_gemm_tc(*bad, p, None) == _abi.FGPE_E_ARG

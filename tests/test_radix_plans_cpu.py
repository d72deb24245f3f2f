"""Radix plans of the size-specialised transforms (cplan in
fortress_b200/csrc/fgpe_fast.cuh) and their position maps.

The column passes and the persistent batch kernel may take plans other than
the handle's (4*4 in place of 8*2, reversed order, radix 16 first), each with
its own position -> frequency map.  This test compiles the library's own
cplan on the host, checks every plan multiplies out to its line length, and
runs a numpy model of the in-place decimation-in-frequency passes (the stride
pattern of ct_pass, a DFT of each radix, twiddles W_N^(n2 r N/BP)) to check
that position p of the result holds frequency f[p] of the map the host builds
(position_map in fgpe_api.cu, restated here)."""
import os
import shutil
import subprocess

import numpy as np
import pytest

CSRC = os.path.join(os.path.dirname(os.path.dirname(os.path.abspath(__file__))), "fortress_b200", "csrc")
SIZES = (128, 192, 256, 384, 512)
PLANS = (0, 1, 2, 3)

PROBE = r"""
#include <cstdio>
#include "fgpe_kernels.cuh"
#include "fgpe_fast.cuh"
int main() {
    const int ns[5] = {128, 192, 256, 384, 512};
    for (int i = 0; i < 5; ++i)
        for (int pv = 0; pv < 4; ++pv) {
            const fgpe::CPlan p = fgpe::cplan(ns[i], pv);
            std::printf("%d %d", ns[i], pv);
            for (int f = 0; f < p.nf; ++f) std::printf(" %d", p.r[f]);
            std::printf("\n");
        }
    return 0;
}
"""


@pytest.fixture(scope="module")
def plans(tmp_path_factory):
    nvcc = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(nvcc):
        pytest.skip("nvcc not available")
    d = tmp_path_factory.mktemp("plans")
    src = d / "probe.cu"
    src.write_text(PROBE)
    exe = d / "probe"
    subprocess.run([nvcc, "-std=c++17", "--expt-relaxed-constexpr", "-gencode", "arch=compute_100a,code=sm_100a",
                    "-I", CSRC, "-o", str(exe), str(src)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    res = {}
    for line in out.strip().splitlines():
        v = [int(t) for t in line.split()]
        res[(v[0], v[1])] = v[2:]
    return res


def position_map(n, radices):
    f = np.empty(n, dtype=int)
    for k in range(n):
        rem, pos, block = k, 0, n
        for r in radices:
            d = rem % r
            rem //= r
            block //= r
            pos += d * block
        f[pos] = k
    return f


def dif_in_place(x, radices):
    n = len(x)
    s = np.array(x, dtype=complex)
    bp = n
    for r in radices:
        si = bp // r
        tstep = n // bp
        for q in range(n // r):
            blk, n2 = divmod(q, si)
            e = blk * bp + n2 + si * np.arange(r)
            v = np.fft.fft(s[e])
            if n2:
                v = v * np.exp(-2j * np.pi * n2 * np.arange(r) * tstep / n)
            s[e] = v
        bp //= r
    return s


def test_plans_multiply_out(plans):
    for n in SIZES:
        for pv in PLANS:
            r = plans[(n, pv)]
            assert int(np.prod(r)) == n, (n, pv, r)
            assert all(x in (2, 3, 4, 5, 8, 16) for x in r), (n, pv, r)


def test_radix16_where_it_saves_a_pass(plans):
    # 128 = 16*8, 256 = 16*16, 384 = 16*8*3; 192 and 512 keep plan 0
    assert plans[(128, 3)] == [16, 8] and plans[(256, 3)] == [16, 16] and plans[(384, 3)] == [16, 8, 3]
    for n in (192, 512):
        assert plans[(n, 3)] == plans[(n, 0)]
    for n in SIZES:
        assert len(plans[(n, 3)]) <= len(plans[(n, 0)])
        assert plans[(n, 2)] == plans[(n, 0)][::-1]


@pytest.mark.parametrize("n", SIZES)
def test_dif_passes_follow_the_position_map(plans, n):
    rng = np.random.default_rng(n)
    x = rng.standard_normal(n) + 1j * rng.standard_normal(n)
    ref = np.fft.fft(x)
    for pv in PLANS:
        r = plans[(n, pv)]
        f = position_map(n, r)
        assert sorted(f) == list(range(n))
        y = dif_in_place(x, r)
        assert np.abs(y - ref[f]).max() <= 1e-12 * np.abs(ref).max(), (n, pv, r)

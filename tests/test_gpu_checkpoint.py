"""Checkpoint/resume (fgpe_checkpoint_save/load): a run interrupted at step N
and resumed from the file in a fresh handle continues bit-identically."""
import numpy as np
import pytest

from tests.helpers import case_params

pytestmark = pytest.mark.gpu

CASES = [
    dict(dim=2, spin=2, n=(64, 48), imag=True, precision="fp64"),
    dict(dim=3, spin=1, n=(16, 16, 24), imag=False, precision="fp32"),
    dict(dim=1, spin=2, n=(256,), imag=True, precision="fp64"),
    dict(dim=2, spin=1, n=(32, 32), imag=True, precision="fp64", no_soc=True),   # projection branch
]


def _state(shape, ms, seed):
    """A smooth blob with seeded amplitude noise and phases."""
    rng = np.random.default_rng(seed)
    axes = np.meshgrid(*[((np.arange(n) - n / 2) / max(n / 4, 1)) for n in shape], indexing="ij")
    g = np.exp(-sum(a ** 2 for a in axes) / 2.0)
    phi = np.repeat(g[..., None], ms, axis=-1) * (1 + 0.05 * rng.standard_normal(shape + (ms,)))
    return phi * np.exp(1j * rng.uniform(-0.4, 0.4, phi.shape))


def _make(F, c):
    kw = case_params((c["dim"], c["spin"], c["imag"], c["n"]))
    if c.get("no_soc"):
        kw["gamma"] = (0.0, 0.0, 0.0)
        kw["mag"] = 0.3
    kw["precision"] = c["precision"]
    return F.Propagator(**kw)


@pytest.mark.parametrize("c", CASES, ids=lambda c: f"{c['dim']}d-s{c['spin']}-{c['precision']}")
def test_resume_is_bit_identical(c, tmp_path):
    import fortress_b200 as F
    a = _make(F, c)
    a.set_state(_state(a.shape, a.ms, 3))
    if c["imag"]:
        a.normt()
    a.step(7)
    path = tmp_path / "run.ckp"
    a.save(path, step=7, user=[1.25, -3.5])
    a.step(9)
    want, want_n = a.state(), a.normc()
    b = _make(F, c)
    st, u = b.load(path)
    assert st == 7 and u[0] == 1.25 and u[1] == -3.5
    b.step(9)
    got, got_n = b.state(), b.normc()
    assert np.array_equal(got, want)
    assert np.array_equal(got_n, want_n)


def test_load_rejects_bad_files(tmp_path):
    import fortress_b200 as F
    c = CASES[0]
    a = _make(F, c)
    a.set_state(_state(a.shape, a.ms, 4))
    path = tmp_path / "a.ckp"
    a.save(path)
    raw = bytearray(path.read_bytes())
    raw[200] ^= 0x01
    bad = tmp_path / "bad.ckp"
    bad.write_bytes(bytes(raw))
    with pytest.raises(F.FgpeError, match="checksum"):
        a.load(bad)
    other = _make(F, dict(c, n=(32, 48)))
    with pytest.raises(F.FgpeError, match="differs"):
        other.load(path)
    with pytest.raises(F.FgpeError):
        a.load(tmp_path / "missing.ckp")

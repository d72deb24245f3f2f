"""fgpe_norms_async (the per-step NORMC read-back) into the three kinds of
destination it accepts: pinned host memory and device memory (written by a
one-warp kernel in the step chain) and pageable host memory (a copy).  Every
per-step record must equal, bit for bit, what the blocking fgpe_norms returns
for that step."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")

pytestmark = pytest.mark.gpu

CASES = [
    # dim, spin, n, d, precision
    (2, 2, (128, 128), (0.2, 0.2), "fp64"),     # size-specialised passes (PDL chain)
    (2, 1, (96, 40), (0.1, 0.3), "fp32"),       # generic passes
    (1, 2, (4096,), (0.01,), "fp64"),           # split 1D passes
]


@pytest.mark.parametrize("dim,spin,n,d,precision", CASES)
def test_norms_async_matches_blocking_read(dim, spin, n, d, precision):
    import fortress_b200 as F
    ms = 2 * spin + 1
    steps = 6
    prop = F.Propagator(dim=dim, spin=spin, n=n, d=d, dt=1e-3, imag_time=False, tau=(100.0, 5.0, 1.0),
                        gamma=(0.5, 0.5, 0.0), precision=precision)
    try:
        rng = np.random.default_rng(5)
        shape = tuple(n) + (1,) * (3 - len(n)) + (ms,)
        x = [np.linspace(-1.0, 1.0, k) * k * dd / 2.0 for k, dd in zip(n, d)]
        g = np.exp(-sum(np.meshgrid(*[xx ** 2 for xx in x], indexing="ij")) / 2.0)
        g = g.reshape(shape[:3])
        phi = np.stack([g * (1 + 0.1 * rng.standard_normal(g.shape)) for _ in range(ms)], axis=-1)
        prop.set_state(phi.astype(complex))
        prop.normt()
        pinned = torch.full((steps, ms), np.nan, dtype=torch.float64).pin_memory()
        dev = torch.full((steps, ms), np.nan, dtype=torch.float64, device="cuda")
        pageable = np.full((steps, ms), np.nan)
        want = np.zeros((steps, ms))
        for k in range(steps):
            prop.step(1, snapshot=False)
            prop.norms_async(pinned.data_ptr() + 8 * ms * k)
            prop.norms_async(dev.data_ptr() + 8 * ms * k)
            prop.norms_async(pageable.ctypes.data + 8 * ms * k)
            want[k] = prop.normc()                  # synchronises the stream
        torch.cuda.synchronize()
        assert np.all(np.isfinite(want)) and np.all(want > 0)
        assert np.array_equal(pinned.numpy(), want)
        assert np.array_equal(dev.cpu().numpy(), want)
        assert np.array_equal(pageable, want)
    finally:
        prop.close()


# fgpe_norms_sink: the step's own last block appends its NORMC to a ring.
SINK_CASES = CASES + [
    (1, 2, (2048,), (0.01,), "fp64"),          # one cluster per call
    (1, 1, (256,), (0.05,), "fp64"),           # single-block 1D kernel
]


@pytest.mark.parametrize("dim,spin,n,d,precision", SINK_CASES)
def test_norms_sink_records_every_step(dim, spin, n, d, precision):
    import fortress_b200 as F
    ms = 2 * spin + 1
    prop = F.Propagator(dim=dim, spin=spin, n=n, d=d, dt=1e-3, imag_time=False, tau=(100.0, 5.0, 1.0),
                        gamma=(0.5, 0.5, 0.0), precision=precision)
    try:
        rng = np.random.default_rng(7)
        shape = tuple(n) + (1,) * (3 - len(n)) + (ms,)
        x = [np.linspace(-1.0, 1.0, k) * k * dd / 2.0 for k, dd in zip(n, d)]
        g = np.exp(-sum(np.meshgrid(*[xx ** 2 for xx in x], indexing="ij")) / 2.0).reshape(shape[:3])
        phi = np.stack([g * (1 + 0.1 * rng.standard_normal(g.shape)) for _ in range(ms)], axis=-1)
        prop.set_state(phi.astype(complex))
        ring = torch.full((64, ms), np.nan, dtype=torch.float64).pin_memory()
        prop.norms_sink(ring.data_ptr(), 64)
        want = np.zeros((5, ms))
        for k in range(5):                          # one step per call: each record bit for bit
            prop.step(1, snapshot=False)
            want[k] = prop.normc()
        torch.cuda.synchronize()
        got = ring.numpy()
        assert np.array_equal(got[:5], want)
        prop.step(40)                               # a multi-step call (graph replay for most steps)
        last = prop.normc()
        torch.cuda.synchronize()
        got = ring.numpy()
        assert np.all(np.isfinite(got[:45])) and np.all(np.isnan(got[45:]))
        assert np.array_equal(got[44], last)
        # a new ring restarts at record 0 and wraps
        dev = torch.full((4, ms), np.nan, dtype=torch.float64, device="cuda")
        prop.norms_sink(dev.data_ptr(), 4)
        for k in range(6):
            prop.step(1, snapshot=False)
        last = prop.normc()
        torch.cuda.synchronize()
        assert np.array_equal(dev.cpu().numpy()[1], last)  # step 6 -> record 5 % 4
        prop.norms_sink(0, 0)
        before = got.copy()
        prop.step(3)
        torch.cuda.synchronize()
        assert np.array_equal(ring.numpy(), before, equal_nan=True)
        with pytest.raises(F.FgpeError):
            prop.norms_sink(np.zeros(5 * ms).ctypes.data, 5)   # pageable memory is refused
    finally:
        prop.close()

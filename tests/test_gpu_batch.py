"""Batched sweeps: one CUDA-graph launch over many ragged instances gives
bitwise the same states as stepping every instance alone (same kernels, same
order of operations), before and after autotuning."""
import numpy as np
import pytest

from tests.helpers import case_params

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    import fortress_b200 as F
    if not F.device_ok():
        pytest.fail("no usable sm_100 device / libfgpe.so not loaded")
    return F


def _instances():
    rng = np.random.default_rng(4)
    out = []
    for k, n in enumerate([(128, 128), (192, 192), (64, 48), (256, 128), (128, 192), (96, 96)]):
        p = case_params((2, 1, 1, n))
        p["gamma"] = tuple(rng.uniform(0, 2, 2))
        p["tau"] = (float(rng.uniform(200, 4000)), float(rng.uniform(-0.05, 0.05) * 2000), 0.0)
        p["alpha"] = (1.0, float(rng.uniform(1, 2)), 1.0)
        p["precision"] = "fp32" if k % 2 else "fp64"
        out.append(p)
    return out


def _guess(p, seed):
    rng = np.random.default_rng(seed)
    nx, ny = p["n"]
    x = (np.arange(nx) - nx / 2) * p["d"][0]
    y = (np.arange(ny) - ny / 2) * p["d"][1]
    g = np.exp(-(x[:, None] ** 2 + p["alpha"][1] * y[None, :] ** 2) / 2.0)
    return np.stack([g * (1 + 0.1 * rng.standard_normal(g.shape)) for _ in range(3)], axis=-1).astype(complex)


def test_batch_equals_individual(F, tmp_path):
    from fortress_b200.batch import Batch
    insts = _instances()
    b = Batch(insts)
    singles = [F.Propagator(**p) for p in insts]
    for i, p in enumerate(insts):
        phi = _guess(p, i)
        b[i].set_state(phi); singles[i].set_state(phi)
        b[i].normt(); singles[i].normt()
    b.config(width=4, steps_per_graph=5)
    b.step(12)                    # graphs of 5, 5 and 2 steps
    for s in singles:
        s.step(12)
    for i in range(len(insts)):
        assert np.array_equal(b[i].state(), singles[i].state())
        assert np.array_equal(b[i].normc(), singles[i].normc())
    obs = b.observables()
    for i, s in enumerate(singles):
        en, mu, mz, rms = s.observables()
        assert obs[i]["en"] == en and np.array_equal(obs[i]["rms"], rms)
        assert obs[i]["conv"] == s.conv()
    # autotuning restores the states it used for its trials
    cache = str(tmp_path / "tune.txt")
    w, k = b.autotune(trial_steps=4, cache_path=cache)
    assert w >= 1 and k >= 2
    b.step(7)
    for s in singles:
        s.step(7)
    for i in range(len(insts)):
        assert np.allclose(b[i].state(), singles[i].state(), rtol=0, atol=1e-13 if insts[i]["precision"] == "fp64" else 1e-6)
    # the cache reproduces the choice
    b2 = Batch(insts)
    for i, p in enumerate(insts):
        b2[i].set_state(_guess(p, i))
    assert b2.autotune(trial_steps=4, cache_path=cache) == (w, k)


def test_timed_batch_step(F):
    """fgpe_batch_step_timed advances like fgpe_batch_step and reports the
    device time of its graph launches; a single-step remainder is refused."""
    from fortress_b200.batch import Batch
    insts = _instances()[:3]
    a, b = Batch(insts), Batch(insts)
    for i, p in enumerate(insts):
        phi = _guess(p, 10 + i)
        for x in (a, b):
            x[i].set_state(phi)
            x[i].normt()
    for x in (a, b):
        x.config(width=2, steps_per_graph=4)
    a.step(10)
    ms = b.step_timed(10)          # graphs of 4, 4 and 2 steps
    assert ms > 0
    for i in range(len(insts)):
        assert np.array_equal(a[i].state(), b[i].state())
    with pytest.raises(F.FgpeError):
        b.step_timed(9)            # 4 + 4 + 1


def _grouped_instances():
    """Two instances per group (128^2 spin-1 FP64 imaginary, 192x128 spin-2
    FP32 real time, 512^2 and 384x256 spin-1 FP64) plus one instance of a
    size the grouped kernels do not cover (on its own branch)."""
    rng = np.random.default_rng(9)
    out = []
    for n, spin, imag, prec in [((128, 128), 1, 1, "fp64"), ((128, 128), 1, 1, "fp64"),
                                ((192, 128), 2, 0, "fp32"), ((192, 128), 2, 0, "fp32"),
                                ((512, 512), 1, 1, "fp64"), ((384, 256), 1, 0, "fp64"),
                                ((384, 256), 1, 0, "fp64"), ((96, 80), 1, 1, "fp64")]:
        p = case_params((2, spin, imag, n))
        p["gamma"] = tuple(rng.uniform(0, 2, 2))
        if spin == 1:
            p["tau"] = (float(rng.uniform(200, 4000)), float(rng.uniform(-0.05, 0.05) * 2000), 0.0)
            if not imag:
                # real time at c0 ~ 4000 from this noisy start is unstable: the
                # oracle amplifies a 1e-15 change of the start to 6e-7 in 12
                # steps, so separately compiled kernels (FMA contraction) could
                # not agree to rounding; a tenth of the coupling grows it to 5e-15
                p["tau"] = (p["tau"][0] / 10, p["tau"][1] / 10, 0.0)
        p["alpha"] = (1.0, float(rng.uniform(1, 2)), 1.0)
        p["d"] = (25.6 / n[0], 25.6 / n[1])
        p["precision"] = prec
        out.append(p)
    return out


def _guess_ms(p, seed):
    ms = 2 * p["spin"] + 1
    g = _guess(p, seed)[..., :1]
    rng = np.random.default_rng(seed + 1)
    return np.concatenate([g * (1 + 0.05 * rng.standard_normal(g.shape)) for _ in range(ms)], axis=-1)


def test_grouped_batch_matches_individual(F):
    """Grouped launches (one pass launch per group of equal grid shapes)
    against each instance stepped alone: the same per-tile arithmetic in
    separately compiled kernels, so the states agree to rounding (the NORMC
    summation order and the compiler's contraction of products into FMAs),
    and NORMC, the observables and CONV agree likewise."""
    from fortress_b200.batch import Batch
    insts = _grouped_instances()
    b = Batch(insts)
    b.mode(grouped=True)
    singles = [F.Propagator(**p) for p in insts]
    for i, p in enumerate(insts):
        phi = _guess_ms(p, 20 + i)
        for x in (b[i], singles[i]):
            x.set_state(phi)
            if p["imag_time"]:
                x.normt()
    b.config(width=4, steps_per_graph=5)
    b.step(12)                    # graphs of 5, 5 and 2 steps
    for s in singles:
        s.step(12)
    obs = b.observables()
    for i, p in enumerate(insts):
        # FP32: a single handle's y pass on 128-point lines takes the radix-16
        # plan, the grouped kernels radix 8*8*2: different FP32 rounding of the
        # transforms, 2.7e-6 of the largest value after the 12 real-time steps
        tol = 1e-13 if p["precision"] == "fp64" else 5e-6
        sa, sb = b[i].state(), singles[i].state()
        assert np.abs(sa - sb).max() <= tol * np.abs(sb).max(), (i, float(np.abs(sa - sb).max()))
        # reductions are FP64 in both precisions, of states that agree to tol
        rt = 1e-12 if p["precision"] == "fp64" else 1e-6
        assert np.allclose(b[i].normc(), singles[i].normc(), rtol=rt, atol=0), i
        en, mu, mz, rms = singles[i].observables()
        assert abs(obs[i]["en"] - en) <= rt * abs(en) and np.allclose(obs[i]["rms"], rms, rtol=rt), i
        assert abs(obs[i]["conv"] - singles[i].conv()) <= (1e-10 if p["precision"] == "fp64" else 1e-4) * \
            max(singles[i].conv(), 1e-12), i

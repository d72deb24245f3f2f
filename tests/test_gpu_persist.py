"""Persistent batch mode: one kernel launch per graph of steps advances every
q2D instance of a size-specialised grid (one launch per spin and precision),
taking work items from a device ticket counter; per-instance device counters
order the passes.  Each kernel variant (tile shapes, radix plan of the y
lines) must give the states of the instances stepped alone, and a device-side
wait that cannot end must come back as FGPE_E_TIMEOUT, not as a hang."""
import numpy as np
import pytest

from tests.test_gpu_batch import _grouped_instances, _guess_ms

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def F():
    import fortress_b200 as F
    if not F.device_ok():
        pytest.fail("no usable sm_100 device / libfgpe.so not loaded")
    return F


def _start(F, insts, b, seed=20):
    singles = [F.Propagator(**p) for p in insts]
    for i, p in enumerate(insts):
        phi = _guess_ms(p, seed + i)
        for x in (b[i], singles[i]):
            x.set_state(phi)
            if p["imag_time"]:
                x.normt()
    return singles


@pytest.mark.parametrize("variant", [0, 1, 2, 3, 4])
def test_persistent_matches_individual(F, variant):
    """Spin-1 FP64 instances of 128^2, 512^2 and 384x256 (imaginary and real
    time) share one launch, the spin-2 FP32 192x128 pair another, and a 96x80
    instance keeps its own branch.  Against each instance stepped alone the
    per-tile arithmetic is the same up to the y radix plan, the NORMC
    summation order and FMA contraction, so states agree to rounding; NORMC,
    the observables and CONV (the last two steps' snapshots) likewise."""
    from fortress_b200.batch import Batch
    insts = _grouped_instances()
    b = Batch(insts)
    b.mode(persistent=True)
    assert b.variant(variant) == variant
    singles = _start(F, insts, b)
    b.config(width=4, steps_per_graph=5)
    b.step(12)                    # launches of 5, 5 and 2 steps
    for s in singles:
        s.step(12)
    obs = b.observables()
    # FP32: the y radix plans differ (a single handle's y pass takes the
    # radix-16 plan on 128-point lines), so the transforms round differently:
    # up to 2.7e-6 of the largest value after the 12 real-time spin-2 steps
    for i, p in enumerate(insts):
        tol = 1e-13 if p["precision"] == "fp64" else 5e-6
        sa, sb = b[i].state(), singles[i].state()
        assert np.abs(sa - sb).max() <= tol * np.abs(sb).max(), (i, float(np.abs(sa - sb).max()))
        rt = 1e-12 if p["precision"] == "fp64" else 1e-6
        assert np.allclose(b[i].normc(), singles[i].normc(), rtol=rt, atol=0), i
        en, mu, mz, rms = singles[i].observables()
        assert abs(obs[i]["en"] - en) <= rt * abs(en) and np.allclose(obs[i]["rms"], rms, rtol=rt), i
        assert abs(obs[i]["conv"] - singles[i].conv()) <= (1e-10 if p["precision"] == "fp64" else 1e-4) * \
            max(singles[i].conv(), 1e-12), i


def test_persistent_timed_and_reused(F):
    """step_timed in persistent mode advances like step, and a second call
    reuses the captured launch (instance tables refreshed, counters cleared
    inside the graph)."""
    from fortress_b200.batch import Batch
    insts = _grouped_instances()[:5]
    a, b = Batch(insts), Batch(insts)
    for x in (a, b):
        x.mode(persistent=True)
        x.config(width=2, steps_per_graph=4)
    _start(F, insts, a, seed=40)
    _start(F, insts, b, seed=40)
    a.step(8)
    a.step(8)
    ms = b.step_timed(16)
    assert ms > 0
    for i in range(len(insts)):
        assert np.array_equal(a[i].state(), b[i].state()), i


def test_persistent_wait_runs_out(F):
    """A row wait that no block can satisfy (test hook) runs out after the
    bound and the step reports FGPE_E_TIMEOUT; the batch then steps normally
    again once its states are set afresh."""
    from fortress_b200 import _abi
    from fortress_b200.batch import Batch
    insts = _grouped_instances()[:4]
    b = Batch(insts)
    b.mode(persistent=True)
    b.config(width=2, steps_per_graph=4)
    singles = _start(F, insts, b, seed=60)
    b.wait_bound(5.0, stall_instance=1)
    with pytest.raises(F.FgpeError) as err:
        b.step(4)
    assert err.value.args[0].startswith(f"fgpe error {_abi.FGPE_E_TIMEOUT}")
    assert "instance 1" in err.value.args[0]
    b.wait_bound(2000.0)
    for i, p in enumerate(insts):
        phi = _guess_ms(p, 60 + i)
        b[i].set_state(phi)
        if p["imag_time"]:
            b[i].normt()
    b.step(4)
    for s in singles:
        s.step(4)
    for i, p in enumerate(insts):
        tol = 1e-13 if p["precision"] == "fp64" else 5e-6   # radix plans as above
        sa, sb = b[i].state(), singles[i].state()
        assert np.abs(sa - sb).max() <= tol * np.abs(sb).max(), i


def test_autotune_covers_persistent_variants(F, tmp_path):
    """The autotuner's search includes the persistent mode with every kernel
    variant; whatever it keeps, stepping afterwards matches the instances
    stepped alone, and the cached choice is reproduced."""
    from fortress_b200.batch import Batch
    insts = _grouped_instances()[:5]
    b = Batch(insts)
    singles = _start(F, insts, b, seed=80)
    cache = str(tmp_path / "tune.txt")
    w, k = b.autotune(trial_steps=4, cache_path=cache)
    v = b.variant()
    line = open(cache).read().split()
    assert int(line[-1]) == v and int(line[-2]) in (0, 1, 2)
    b.step(6)
    for s in singles:
        s.step(6)
    for i, p in enumerate(insts):
        tol = 1e-13 if p["precision"] == "fp64" else 5e-6   # any y plan (see above)
        sa, sb = b[i].state(), singles[i].state()
        assert np.abs(sa - sb).max() <= tol * np.abs(sb).max(), i
    b2 = Batch(insts)
    _start(F, insts, b2, seed=80)
    assert b2.autotune(trial_steps=4, cache_path=cache) == (w, k) and b2.variant() == v

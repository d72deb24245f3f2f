"""What the trained 3D network gains over the method without it, on a
reduced grid: ground states of the 3D spin-1 parameter box (fortress_b200.
fno3d.BOX3) computed by the solver on a 32^3 grid of the 25.6 box, a small
network trained on them with the library's kernels, and, for held-out
parameter points, the guess it gives against INITIALIZE's Gaussian
(cgpe3d.f90:783-785), the start the reference uses.

The gain asserted is the one that holds at this scale: the learned start's
energy error |E0 - E*| is at most half the Gaussian's (one measured point:
66 against 191, with 40 training epochs).  The FP64
imaginary-time steps until |E - E*| <= 1e-8 |E*| holds for good are
reported for both starts, not asserted: a guess a few per cent off still
has to let the slow long-wavelength spin mode decay, and a small network's
guess can settle into a nearby higher state (the 256^3 experiment of
fortress_b200.experiments.time_to_gs measures the step gain at full size).
The plain solver from the Gaussian reaches E*, the judge of the guess."""
import numpy as np
import pytest

torch = pytest.importorskip("torch")
pytestmark = pytest.mark.gpu

N = 32
STP = 100


def _steps_to(trace, e_star, tol=1e-8):
    out = None
    for st, en in trace:
        ok = abs(en - e_star) <= tol * abs(e_star)
        if ok and out is None:
            out = st
        elif not ok:
            out = None
    return out


def _run(prop, max_steps):
    trace = [(0, prop.observables()[0])]
    done = 0
    while done < max_steps:
        prop.step(STP)
        done += STP
        trace.append((done, prop.observables()[0]))
    return trace


def test_learned_guess_starts_closer_to_the_ground_state():
    import fortress_b200 as F
    from fortress_b200 import fno3d as F3
    from fortress_b200.experiments import time_to_gs as T
    pts = T.box_points(24, seed=5)
    held = T.box_points(2, seed=6)
    states, conv = T.ground_states(pts, N, 20000, precision="fp32", chunk=24)
    assert np.all(np.isfinite(states))
    net, hist = T.train(pts, states, N, epochs=80, batch=4, lr=3e-3, width=8, modes=6, layers=3, hidden=32)
    assert hist[-1] < 0.2 * hist[0], hist
    infer = F3.FNO3(N, 1, params=net.params_numpy(), width=8, modes=6, layers=3, hidden=32, train=False)
    for pt in held:
        p = T.params(pt, N, "fp64")
        a = F.Propagator(**p)
        a.set_state(T.gaussian_start(N))
        a.normt()
        ta = _run(a, 60000)
        a.close()
        guess = T.learned_guess_device(infer, pt, N)
        b = F.Propagator(**p)
        b.set_state_device(guess.data_ptr())
        b.normt()
        tb = _run(b, 60000)
        b.close()
        e_star = min(ta[-1][1], tb[-1][1])
        err_g, err_l = abs(ta[0][1] - e_star), abs(tb[0][1] - e_star)
        print({"point": pt.tolist(), "E*": e_star, "E0_error_gaussian": err_g, "E0_error_learned": err_l,
               "steps_gaussian": _steps_to(ta, e_star), "steps_learned": _steps_to(tb, e_star)})
        assert err_l <= 0.5 * err_g, (err_l, err_g)
        assert _steps_to(ta, ta[-1][1]) is not None

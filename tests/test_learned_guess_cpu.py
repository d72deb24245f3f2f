"""Host-side pieces of the learned-guess experiment (no device needed)."""
import numpy as np

from fortress_b200 import fno as FN
from fortress_b200.experiments import learned_guess as LG


def test_parameter_box_and_instances():
    rows = LG.box(50, 5)
    assert rows.shape == (50, 5)
    assert np.all((rows[:, :2] >= 0) & (rows[:, :2] <= 2))
    assert np.all((rows[:, 2] >= 100) & (rows[:, 2] <= 2000))
    assert np.all(np.abs(rows[:, 3]) <= 0.05) and np.all((rows[:, 4] >= 1) & (rows[:, 4] <= 2))
    np.testing.assert_array_equal(rows, LG.box(50, 5))            # seeded
    p = LG.instance(rows[0], 64)
    assert p["d"] == (0.4, 0.4) and p["tau"][0] == 2 * rows[0, 2]
    assert abs(p["tau"][1] - 2 * rows[0, 2] * rows[0, 3]) < 1e-12
    pn = FN.normalise_params(*rows.T)
    assert np.all(np.abs(pn) <= 1.0 + 1e-12)


def test_target_round_trip_and_inputs():
    rng = np.random.default_rng(0)
    states = [rng.standard_normal((8, 8, 3)) + 1j * rng.standard_normal((8, 8, 3)) for _ in range(3)]
    back = LG.target_to_states(LG.states_to_target(states))
    for a, b in zip(states, back):
        np.testing.assert_allclose(a, b, rtol=1e-6, atol=1e-6)
    a = FN.input_channels(rng.uniform(-1, 1, (3, 5)), 16)
    assert a.shape == (7, 3, 16, 16)
    assert a[5, 0, 0, 0] == -1.0 and a[6, 0, 0, 1] == -1.0 + 2.0 / 16


def test_first_within():
    e_star = np.array([1.0, 2.0])
    traj = np.array([[1.5, 2.0], [1.0, 2.5], [1.0, 2.0], [1.0, 2.0]])
    got = LG.first_within(traj, 100, e_star, 1e-8)
    np.testing.assert_array_equal(got, [200, 300])

"""The DA-ray retirement policy of the surrogate (host logic, no GPU)."""
import numpy as np

from simtrack_b200.surrogate import ray_policy


def test_ray_policy_rules():
    namp = 14
    # ray 0: lost early from amplitude 9; the classifier calls everything below stable
    # ray 1: nothing lost early; the classifier calls amplitude 7 lost, amplitude 2 uncertain
    lost = np.zeros((2, namp), dtype=bool)
    lost[0, 9:11] = True
    p = np.full((2, namp), 0.999)
    p[0, 9:11] = np.nan
    p[1, 7] = 0.2
    p[1, 2] = 0.7
    retire, stable = ray_policy(lost.ravel(), p.ravel(), namp, 0.99, 2, 2)
    retire, stable = retire.reshape(2, namp), stable.reshape(2, namp)
    # ray 0: band [7, 11] around the known loss at 9; above 9 retired (exact), not as stable;
    # below the band confident -> retired as stable; lost-early particles are never retired
    assert list(retire[0]) == [True] * 7 + [False] * 4 + [True] * 3
    assert list(stable[0]) == [True] * 7 + [False] * 7
    # ray 1: band [5, 9] around the predicted loss at 7; 2 uncertain -> tracked;
    # above the band retired as stable only when confident (the predicted loss may be wrong)
    assert list(retire[1]) == [True, True, False, True, True] + [False] * 5 + [True] * 4
    assert np.array_equal(retire[1], stable[1])


def test_ray_policy_never_retires_predicted_losses():
    namp = 10
    lost = np.zeros(namp, dtype=bool)
    p = np.full(namp, 0.001)  # confidently lost everywhere
    retire, stable = ray_policy(lost, p, namp, 0.99, 1, 1)
    assert not retire.any() and not stable.any()


def test_replay_on_saved_experiment():
    """The trained network's outputs on the 32 held-out seeds (seeds 33-64,
    1,760 DA rays, saved by `python -m simtrack_b200.surrogate --artifacts`):
    with the default policy every ray's DA equals the plain 1e5-turn scan's
    while ~18 % of the particles alive at turn 1,024 stay tracked."""
    from pathlib import Path

    from simtrack_b200.surrogate import replay_policies
    path = Path(__file__).resolve().parents[1] / "simtrack_b200" / "data" / "surrogate_rhic_like.npz"
    rows = replay_policies(str(path), confidences=(0.99,), bands=((2, 2),))
    assert rows[0]["rays_differing"] == 0
    assert rows[0]["tracked_to_end"] < 0.2 * 63851

"""What the trained surrogate gains over the plain scan (needs a B200).

A small version of the surrogate-pruned DA scan: train on four error seeds,
evaluate on two held-out seeds, and compare with the plain scan of the same
seeds: the pruned scan must track far fewer particle-turns while giving the
same DA per ray within one amplitude step, and the audited particles must be
classified correctly."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def test_surrogate_prunes_with_matching_da(native_lib):
    from simtrack_b200.surrogate import SurrogateConfig, experiment
    cfg = SurrogateConfig(nturn=6144, nrec=1024, window=512, epochs=80, audit=0.05, batch=1024)
    namp, amax = 24, 12.0
    res = experiment([1, 2, 3, 4], [5, 6], namp=namp, amax=amax, nang=4, deltas=(0.0, 6e-4), cfg=cfg,
                     log=lambda *a: None)
    step = amax / (namp - 1)
    # the gain: a large share of the survivors stops at turn 1024
    assert res["pruned"]["retired"] > 0.3 * res["pruned"]["alive_at_nrec"]
    assert res["speedup_particle_turns"] > 1.5
    # the DA barely moves: within one grid step on every ray
    assert res["da_error_sigma"]["max"] <= step + 1e-9
    assert res["pruned"]["audit_accuracy"] > 0.95

"""Checkpoint and resume of the learned-colour training state
(splat_cuda_learner_save_state / _load_state): parameters, latents, their
Adam moments, the latent rows' stamps and the step count.

* The state round-trips bit for bit (save -> load into a fresh learner ->
  save gives the same bytes).
* Training resumed from a checkpoint follows the uninterrupted run step for
  step: the same step counts, per-call losses and parameters, up to the
  summation order of the gradient atomics (which differs between any two
  runs, resumed or not).
* A state of another configuration is rejected.
"""

import numpy as np
import pytest

from splat_b200 import _native as N
from splat_b200.render import CudaRenderer
from tests import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def sh_scene(cuda_lib):
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    r = CudaRenderer(scenes.clusters(5000, seed=21, sh_degree=3))
    yield r
    r.close()


def _close_fraction(a, b):
    return float(np.mean(np.isclose(a, b, rtol=2e-3, atol=2e-5)))


def test_resumed_training_matches_uninterrupted(sh_scene):
    from splat_b200.learned import LearnConfig, Learner

    cfg = LearnConfig(directions=32, batch=8192, seed=9)
    a = Learner(sh_scene, cfg)
    b = Learner(sh_scene, cfg)
    c = Learner(sh_scene, cfg)
    try:
        a.train(5)
        state = a.save_state()
        assert len(state) == N.lib().splat_cuda_learner_state_bytes(a._h)
        b.load_state(state)
        assert b.save_state() == state, "the state does not round-trip"
        # Uninterrupted: a trains on; resumed: b trains the same steps from the checkpoint.
        ra = [a.train(3) for _ in range(3)]
        rb = [b.train(3) for _ in range(3)]
        assert [s.steps for s in ra] == [s.steps for s in rb] == [8, 11, 14]
        for sa, sb in zip(ra, rb):
            assert abs(sa.mean_loss - sb.mean_loss) <= 1e-3 * abs(sa.mean_loss)
        pa, la = a.params()
        pb, lb = b.params()
        assert _close_fraction(pa, pb) > 0.995 and _close_fraction(la, lb) > 0.995
        # c trains 14 steps in one go from the start: the same place.
        c.train(14)
        pc, lc = c.params()
        assert _close_fraction(pa, pc) > 0.99 and _close_fraction(la, lc) > 0.99
    finally:
        for x in (a, b, c):
            x.close()


def test_state_of_another_configuration_is_rejected(sh_scene):
    from splat_b200.learned import LearnConfig, Learner

    a = Learner(sh_scene, LearnConfig(directions=32, batch=8192, seed=9))
    other = Learner(sh_scene, LearnConfig(directions=32, batch=8192, seed=10))
    try:
        state = a.save_state()
        with pytest.raises(N.SplatError) as e:
            other.load_state(state)
        assert e.value.code == N.SPLAT_ERR_INVALID_ARG
        with pytest.raises(N.SplatError):
            a.load_state(state[:100])
        with pytest.raises(N.SplatError):
            a.load_state(b"X" * len(state))
        a.load_state(state)  # the learner itself still loads it
    finally:
        a.close()
        other.close()

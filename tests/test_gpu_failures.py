"""Failure detection without a GPU fault (SPLAT_OPT_INJECT_FAULT).

* An allocation that fails (injected on the host: the allocator is not
  called) returns SPLAT_ERR_OOM, and the handle renders afterwards exactly
  as before.
* A tensor-core wait that never completes (injected as a second wait, on an
  mbarrier nothing arrives on, bounded to a few milliseconds) makes the
  learned-colour frame and the training call return SPLAT_ERR_TIMEOUT; the
  kernels free their tensor memory on the way out, a training step that gave
  up is dropped (parameters and step count unchanged), and the next call runs
  normally with the same results as before.

Nothing here faults, traps or hangs the GPU: every wait is bounded, and the
real MMA completions are still waited for before tensor memory is freed.
"""

import numpy as np
import pytest

from splat_b200 import Frame, OrbitCamera, UpAxis
from splat_b200 import _native as N
from splat_b200.render import CudaRenderer
from tests import scenes

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module", autouse=True)
def _gpu(cuda_lib):
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"


def _view(s):
    c, r = s.bounds()
    return OrbitCamera.new(c, r, UpAxis.NEG_Y).view()


def test_injected_allocation_failure_reports_oom_and_recovers():
    s = scenes.clusters(8000, seed=3, sh_degree=1)
    v = _view(s)
    r = CudaRenderer(s)
    try:
        want = Frame()
        r.render(v, 320, 180, (0.0, 0.0, 0.0), want)
        r.set_option(N.SPLAT_OPT_INJECT_FAULT, N.SPLAT_FAULT_ALLOC)
        assert r.get_option(N.SPLAT_OPT_INJECT_FAULT) == N.SPLAT_FAULT_ALLOC
        # A larger frame needs new per-frame buffers: the first allocation fails.
        with pytest.raises(N.SplatError) as e:
            r.render(v, 1280, 720, (0.0, 0.0, 0.0), Frame())
        assert e.value.code == N.SPLAT_ERR_OOM
        assert r.get_option(N.SPLAT_OPT_INJECT_FAULT) == 0, "the injection fires once"
        big = Frame()
        r.render(v, 1280, 720, (0.0, 0.0, 0.0), big)
        again = Frame()
        r.render(v, 320, 180, (0.0, 0.0, 0.0), again)
        assert np.array_equal(again.pixels, want.pixels)
        # Pair-buffer growth absorbs a failed allocation (a smaller capacity, or windows).
        r.set_option(N.SPLAT_OPT_PAIR_CAPACITY, 1024)
        r.set_option(N.SPLAT_OPT_INJECT_FAULT, N.SPLAT_FAULT_ALLOC)
        grown = Frame()
        r.render(v, 320, 180, (0.0, 0.0, 0.0), grown)
        assert np.array_equal(grown.pixels, want.pixels)
    finally:
        r.close()


def test_injected_lost_completion_times_out_a_learned_frame():
    from splat_b200.learned import learned_renderer

    s = scenes.clusters(6000, seed=4, sh_degree=0)
    v = _view(s)
    rng = np.random.default_rng(5)
    lat = rng.normal(0, 0.6, (len(s), 16)).astype(np.float16).view(np.uint16)
    prm = (rng.normal(0, 0.2, N.MLP_PARAMS)).astype(np.float16).view(np.uint16)
    r = learned_renderer(s.to_fp16(), lat, prm)
    try:
        want = Frame()
        r.render(v, 320, 180, (0.0, 0.0, 0.0), want)
        for _ in range(2):  # twice: the handle and the tensor memory stay usable
            r.set_option(N.SPLAT_OPT_INJECT_FAULT, N.SPLAT_FAULT_LOST_WAIT | (2000 << 8))
            with pytest.raises(N.SplatError) as e:
                r.render(v, 320, 180, (0.0, 0.0, 0.0), Frame())
            assert e.value.code == N.SPLAT_ERR_TIMEOUT
            got = Frame()
            r.render(v, 320, 180, (0.0, 0.0, 0.0), got)
            assert np.array_equal(got.pixels, want.pixels)
    finally:
        r.close()


def test_injected_lost_completion_drops_a_training_step():
    from splat_b200.learned import LearnConfig, Learner

    s = scenes.clusters(4000, seed=6, sh_degree=3)
    sh = CudaRenderer(s)
    learner = Learner(sh, LearnConfig(directions=16, batch=4096, seed=3))
    try:
        p0, l0 = learner.params()
        learner.set_option(N.SPLAT_OPT_INJECT_FAULT, N.SPLAT_FAULT_LOST_WAIT | (2000 << 8))
        with pytest.raises(N.SplatError) as e:
            learner.train(1)
        assert e.value.code == N.SPLAT_ERR_TIMEOUT
        p1, l1 = learner.params()
        assert np.array_equal(p0, p1) and np.array_equal(l0, l1), "a dropped step must not update"
        st = learner.train(2)
        assert st.steps == 2, "the dropped step is not counted"
        p2, _ = learner.params()
        assert not np.array_equal(p0, p2)
        # The same two steps on a fresh learner give the same parameters, up to
        # the order of the gradient atomics (a near-zero gradient sum may flip
        # sign, and Adam's first steps move by +-lr whatever its size).
        fresh = Learner(sh, LearnConfig(directions=16, batch=4096, seed=3))
        fresh.train(2)
        pf, _ = fresh.params()
        fresh.close()
        assert np.mean(np.isclose(p2, pf, rtol=1e-3, atol=1e-5)) > 0.995
    finally:
        learner.close()
        sh.close()

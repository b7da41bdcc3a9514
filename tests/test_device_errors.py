"""Device-side error paths, made to fire without a fault: the reference exits the process on
any CUDA error (gpuAssert, include/macro_helper.h:10-19); here a kernel that hits a limit sets
an error flag and returns, the call reports PT_ERR_DEVICE and the session keeps working.

  * traversal stack: a query that needs more stack entries than it has gives up (the frame's
    kernels, pt_trace_rays, pt_occluded), capped below the BVH depth by the test hook;
  * tensor-core inference: the first wait of each tcgen05 layer limited to one non-blocking
    poll gives up while the MMA runs; the bounded drain still waits for that MMA before the
    kernel frees tensor memory.
Nothing here traps, faults or hangs: every wait is bounded and every access stays in the
stack the kernel was launched with."""
import numpy as np
import pytest

import pathed
from _util import seeded_rays


@pytest.mark.gpu
def test_host_rejects_bad_limits():
    s = pathed.Session(8, 8)
    with pytest.raises(pathed.PathedError) as e:
        s.set_test_limits(-1, 0)
    assert e.value.code == pathed.PT_ERR_ARG
    s.close()


@pytest.mark.gpu
def test_traversal_stack_overflow_is_reported_and_recoverable():
    s = pathed.Session(64, 36)
    s.load_config(2, level=4)
    assert s.counts().bvh_depth >= 4
    s.render(2)
    ref = s.readback().copy()
    sc = s.export_scene()
    o, d, tmin, tmax = seeded_rays(sc, 4000, seed=5)
    ok = s.trace_rays(o, d, tmin, tmax)
    s.set_test_limits(stack_entries=1)
    s.reset()
    with pytest.raises(pathed.PathedError) as e:
        s.render(2)
    assert e.value.code == pathed.PT_ERR_DEVICE and "stack" in str(e.value)
    with pytest.raises(pathed.PathedError) as e:
        s.trace_rays(o, d, tmin, tmax)
    assert e.value.code == pathed.PT_ERR_DEVICE
    with pytest.raises(pathed.PathedError) as e:
        s.occluded(o, d, tmin, tmax)
    assert e.value.code == pathed.PT_ERR_DEVICE
    # limit off: the next calls run normally and give the same results as before
    s.set_test_limits(0, 0)
    s.reset()
    s.render(2)
    assert np.array_equal(s.readback(), ref)
    again = s.trace_rays(o, d, tmin, tmax)
    for k in ("prim_type", "prim_id", "mat_id", "t"):
        assert np.array_equal(again[k], ok[k])
    s.close()


@pytest.mark.gpu
def test_tensor_core_wait_limit_is_reported_and_recoverable():
    from test_guide import random_batch, random_params

    s = pathed.Session(8, 8)
    s.set_guide_params(random_params(21))
    s.set_guide_inference(True)
    x, _, _ = random_batch(3000, seed=22)
    ref = s.guide_forward(x).copy()
    s.set_test_limits(mma_polls=1)
    with pytest.raises(pathed.PathedError) as e:
        s.guide_forward(x)
    assert e.value.code == pathed.PT_ERR_DEVICE and "tensor-core" in str(e.value)
    s.set_test_limits(0, 0)
    assert np.array_equal(s.guide_forward(x), ref)
    s.close()


@pytest.mark.gpu
def test_guided_frame_reports_the_tensor_core_wait_limit():
    """the same limit inside a guided frame: pt_render (through pt_wait) returns
    PT_ERR_DEVICE, the frame after it renders normally"""
    s = pathed.Session(64, 64)
    s.load_config(3, level=3)
    s.set_guiding(True)
    s.set_guide_inference(True)
    s.set_guide_options(steps_per_frame=2, warmup_steps=2)
    for _ in range(4):  # past the warm-up: frames sample the guide (inference runs)
        s.render(1)
    assert s.guide_info()["mode"] == 2
    s.set_test_limits(mma_polls=1)
    with pytest.raises(pathed.PathedError) as e:
        s.render(1)
    assert e.value.code == pathed.PT_ERR_DEVICE
    s.set_test_limits(0, 0)
    s.render(1)
    assert np.all(np.isfinite(s.readback()))
    s.close()

"""pt_trace_rays_static: closest-hit queries that allocate nothing.

Some callers cannot call cudaMalloc: cudaMalloc/cudaFree may synchronize the device (an
interactive pick while a frame renders would stall), and a host whose device memory belongs
to its own allocator has none to hand out. This entry point stages rays and results through
a fixed file-scope device array instead, on a stream of its own. It must return exactly what
pt_trace_rays returns, call after call (the array is reused and keeps the previous call's
contents), leave the device's free memory unchanged, and answer while a frame is in flight.

This file is collected last on purpose, so a run that stops at the first failure has run
every other test before it.
"""
import ctypes as C

import numpy as np
import pytest

import pathed
from _util import seeded_rays


def _static(s, o, d, tmin, tmax, bary=True):
    n = o.shape[0]
    out = {"prim_type": np.empty(n, np.int32), "prim_id": np.empty(n, np.int32), "mat_id": np.empty(n, np.int32),
           "t": np.empty(n, np.float32)}
    if bary:
        out["bary"] = np.empty((n, 2), np.float32)
    rc = pathed.lib.pt_trace_rays_static(s._h, o.ctypes.data, d.ctypes.data, tmin.ctypes.data, tmax.ctypes.data, n,
                                         out["prim_type"].ctypes.data, out["prim_id"].ctypes.data,
                                         out["mat_id"].ctypes.data, out["t"].ctypes.data,
                                         out["bary"].ctypes.data if bary else None)
    return rc, out


@pytest.mark.gpu
@pytest.mark.parametrize("cfg,level", [(1, None), (3, 4)])
def test_static_entry_matches_allocating_entry(cfg, level):
    s = pathed.Session(32, 32)
    s.load_config(cfg, level=level)
    sc = s.export_scene()
    o1, d1, tmin1, tmax1 = seeded_rays(sc, 20000, seed=21)
    o2, d2, tmin2, tmax2 = seeded_rays(sc, 7000, seed=22)  # second call: fewer rays, other rays
    # scene not yet on the device: the static entry must refuse rather than allocate
    rc, _ = _static(s, o1, d1, tmin1, tmax1)
    assert rc == pathed.PT_ERR_STATE
    ref1 = s.trace_rays(o1, d1, tmin1, tmax1, with_bary=True)  # allocating call uploads the scene
    ref2 = s.trace_rays(o2, d2, tmin2, tmax2, with_bary=True)
    for (o, d, tmin, tmax), ref in (((o1, d1, tmin1, tmax1), ref1), ((o2, d2, tmin2, tmax2), ref2)):
        for bary in (True, False):  # with and without the barycentrics copy
            rc, got = _static(s, o, d, tmin, tmax, bary)
            assert rc == pathed.PT_OK, pathed.lib.pt_last_error(s._h)
            for k in got:
                assert np.array_equal(got[k], ref[k]), k  # bit-exact, the tolerance of the other trace tests
    # an edit leaves the device copy stale: refused until an allocating call uploads it again
    s.set_material(0, pathed.LAMBERTIAN, albedo=(0.5, 0.5, 0.5))
    rc, _ = _static(s, o2, d2, tmin2, tmax2)
    assert rc == pathed.PT_ERR_STATE
    ref3 = s.trace_rays(o2, d2, tmin2, tmax2, with_bary=True)
    rc, got = _static(s, o2, d2, tmin2, tmax2)
    assert rc == pathed.PT_OK and all(np.array_equal(got[k], ref3[k]) for k in got)
    s.close()


@pytest.mark.gpu
def test_static_entry_allocates_nothing():
    """free device memory is the same before and after static calls of different sizes"""
    import torch

    s = pathed.Session(32, 32)
    s.load_config(1)
    sc = s.export_scene()
    o, d, tmin, tmax = seeded_rays(sc, 30000, seed=5)
    s.trace_rays(o[:16], d[:16], tmin[:16], tmax[:16])  # uploads the scene (allocating)
    assert _static(s, o[:8], d[:8], tmin[:8], tmax[:8])[0] == pathed.PT_OK  # first call: address look-up
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    for n in (30000, 100, 65536 // 2, 1):
        rc, _ = _static(s, o[:n], d[:n], tmin[:n], tmax[:n], bary=n % 2 == 0)
        assert rc == pathed.PT_OK
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0, f"free device memory changed by {free0 - free1} bytes"
    s.close()


@pytest.mark.gpu
def test_static_entry_while_a_frame_is_in_flight():
    """a query made between pt_render_async and pt_wait runs on the session's query stream and
    returns the same hits as after the frame"""
    s = pathed.Session(512, 512)
    s.load_config(1)
    sc = s.export_scene()
    o, d, tmin, tmax = seeded_rays(sc, 20000, seed=8)
    ref = s.trace_rays(o, d, tmin, tmax, with_bary=True)
    s.render(1)  # frame buffers and graph set up
    s.render_async(32)
    rc, got = _static(s, o, d, tmin, tmax)
    done = C.c_int(0)
    pathed.lib.pt_poll(s._h, C.byref(done), None)
    print(f"frame still in flight when the static query returned: {done.value == 0}")
    s.wait()
    assert rc == pathed.PT_OK, pathed.lib.pt_last_error(s._h)
    for k in got:
        assert np.array_equal(got[k], ref[k]), k
    s.close()


@pytest.mark.gpu
def test_static_entry_limits():
    s = pathed.Session(16, 16)
    s.load_config(0)
    sc = s.export_scene()
    o, d, tmin, tmax = seeded_rays(sc, 64, seed=1)
    s.trace_rays(o, d, tmin, tmax)
    n = pathed.STATIC_MAX_RAYS + 1
    big = np.zeros((n, 3), np.float32)
    rc = pathed.lib.pt_trace_rays_static(s._h, big.ctypes.data, big.ctypes.data, big.ctypes.data, big.ctypes.data, n,
                                         big.ctypes.data, big.ctypes.data, big.ctypes.data, big.ctypes.data, None)
    assert rc == pathed.PT_ERR_ARG
    assert b"PT_STATIC" in pathed.lib.pt_last_error(s._h) or b"ray count" in pathed.lib.pt_last_error(s._h)
    rc, got = _static(s, o[:0], d[:0], tmin[:0], tmax[:0])
    assert rc == pathed.PT_OK
    s.close()

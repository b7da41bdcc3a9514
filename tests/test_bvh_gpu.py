"""GPU BVH builders (a Morton-order LBVH, or PLOC clustering, collapsed to the wide node
format): their trees pass the host builder's structural check, and the closest hits and
images they give are identical to those of the host's binned-SAH trees (the tie rule lives in
the leaf test; the padding keeps every child box conservative)."""
import numpy as np
import pytest

import pathed
from _util import seeded_rays


def _session(config, level, width, leaf, gpu, w=64, h=64):
    s = pathed.Session(w, h)
    s.set_bvh_builder(gpu)
    s.load_config(config, level=level)
    s.set_bvh(width, leaf)
    return s


def test_gpu_builder_defers_the_build():
    s = _session(2, 3, 4, 4, True)
    c = s.counts()
    assert c.num_triangles == 20 * 4 ** 3
    assert c.bvh_nodes == 0  # built on the device at the first upload
    s.set_bvh_builder(False)  # switching back builds on the host at once
    assert s.counts().bvh_nodes > 0
    assert s.check_bvh() == 0
    s.set_bvh_builder(2)  # PLOC: deferred as well
    assert s.counts().bvh_nodes == 0
    for bad in (-1, 3):
        with pytest.raises(pathed.PathedError) as e:
            s.set_bvh_builder(bad)
        assert e.value.code == pathed.PT_ERR_ARG
    s.close()


CASES = [(0, None, 4, 4), (1, None, 8, 4), (1, None, 2, 1), (2, 4, 4, 4), (3, 3, 8, 16), (2, 5, 2, 2)]


@pytest.mark.gpu
@pytest.mark.parametrize("config,level,width,leaf", CASES)
@pytest.mark.parametrize("builder", [1, 2], ids=["lbvh", "ploc"])
def test_gpu_bvh_same_hits_as_host_bvh(config, level, width, leaf, builder):
    g = _session(config, level, width, leaf, builder)
    h = _session(config, level, width, leaf, False)
    sc = h.export_scene()
    o, d, tmin, tmax = seeded_rays(sc, 20000, seed=config + 7 * width)
    rg = g.trace_rays(o, d, tmin, tmax)
    rh = h.trace_rays(o, d, tmin, tmax)
    for k in ("prim_type", "prim_id", "mat_id", "t"):
        assert np.array_equal(rg[k], rh[k]), k
    assert g.check_bvh() == 0  # every primitive once, inside all its ancestors' boxes
    cg, ch = g.counts(), h.counts()
    assert cg.bvh_width == width and 1 <= cg.bvh_max_leaf <= leaf and cg.bvh_nodes > 0
    print(f"config {config}: GPU tree ({builder}) {cg.bvh_nodes} nodes depth {cg.bvh_depth}; "
          f"host tree {ch.bvh_nodes} nodes depth {ch.bvh_depth}")
    g.close()
    h.close()


@pytest.mark.gpu
def test_gpu_bvh_renders_the_same_image():
    imgs = []
    for gpu in (1, 2, 0):
        s = _session(3, 4, 4, 4, gpu, 96, 96)
        s.set_seed(5)
        for _ in range(2):
            s.render(4)
        imgs.append(s.readback())
        s.close()
    assert np.array_equal(imgs[0], imgs[1]) and np.array_equal(imgs[0], imgs[2])


@pytest.mark.gpu
@pytest.mark.parametrize("builder", [1, 2], ids=["lbvh", "ploc"])
def test_gpu_bvh_build_time_on_the_large_mesh(builder):
    """configuration 2's 1,310,720-triangle mesh: the device build, timed with events"""
    g = _session(2, None, 4, 4, builder)
    g.render(1)
    cg = g.counts()
    h = _session(2, None, 4, 4, False)
    ch = h.counts()
    print(f"BVH build: GPU ({builder}) {cg.bvh_build_ms:.1f} ms ({cg.bvh_nodes} nodes, depth {cg.bvh_depth}), "
          f"host SAH {ch.bvh_build_ms:.1f} ms ({ch.bvh_nodes} nodes, depth {ch.bvh_depth})")
    assert cg.bvh_build_ms > 0
    assert g.check_bvh() == 0
    g.close()
    h.close()

"""Quantized wide BVH nodes (pt_set_bvh_nodes): 8-bit child planes relative to a per-node
origin and power-of-two scale, rounded outward at build time. The decoded boxes contain the
float boxes, so every closest hit, and therefore every rendered image, must be identical to
the float-node traversal's (and to the reference scan's)."""
import numpy as np
import pytest

import oracle as orc
import pathed
from _util import seeded_rays

CASES = [(0, None), (1, None), (2, 4), (3, 4)]


def _session(config, level, width, w=64, h=64):
    s = pathed.Session(w, h)
    s.load_config(config, level=level)
    s.set_bvh(width, 4)
    return s


def test_quantized_setting_is_host_state():
    s = _session(0, None, 4)
    s.set_bvh_quantized(True)
    s.set_bvh_quantized(False)
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"cfg{c[0]}")
@pytest.mark.parametrize("width", [4, 8])
def test_quantized_closest_hits_match_reference_scan(case, width):
    s = _session(*case, width)
    sc = s.export_scene()
    O = orc.Oracle()
    o, d, tmin, tmax = seeded_rays(sc, 20000, seed=5 + width)
    ref = O.trace(O.scene(sc), o, d, tmin, tmax)
    s.set_bvh_quantized(True)
    g = s.trace_rays(o, d, tmin, tmax)
    for k in ("prim_type", "prim_id", "mat_id", "t"):
        assert np.array_equal(g[k], ref[k]), k
    assert s.check_bvh() == 0  # every decoded box contains its float box
    occ_q = s.occluded(o, d, tmin, tmax)
    s.set_bvh_quantized(False)
    assert np.array_equal(occ_q, s.occluded(o, d, tmin, tmax))
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("case", CASES, ids=lambda c: f"cfg{c[0]}")
def test_quantized_frames_render_the_same_image(case):
    """the wavefront's own extend and shadow kernels (their quantized instantiations)"""
    imgs, stats = [], []
    for q in (False, True):
        s = _session(*case, 8, 96, 96)
        s.set_bvh_quantized(q)
        s.set_seed(3)
        s.set_profiling(stage_timing=True, work_counters=True)
        for _ in range(2):
            s.render(4)
        imgs.append(s.readback())
        p = s.profile()
        stats.append((s.stats()["rays_extend"], s.stats()["rays_shadow"], p["node_bytes"], p["extend_nodes"]))
        s.close()
    assert np.array_equal(imgs[0], imgs[1])
    assert stats[0][:2] == stats[1][:2]
    assert (stats[0][2], stats[1][2]) == (256, 96)
    # quantized boxes are looser: a few more node visits, far fewer bytes per visit
    assert stats[0][3] <= stats[1][3] <= 1.3 * stats[0][3]
    print(f"config {case[0]}: node visits float {stats[0][3]} quantized {stats[1][3]}")


@pytest.mark.gpu
def test_quantized_full_size_mesh_and_batch():
    s = _session(2, None, 8)
    sc = s.export_scene()
    o, d, tmin, tmax = seeded_rays(sc, 50000, seed=21)
    f = s.trace_rays(o, d, tmin, tmax)
    s.set_bvh_quantized(True)
    q = s.trace_rays(o, d, tmin, tmax)
    for k in ("prim_type", "prim_id", "t"):
        assert np.array_equal(f[k], q[k]), k
    assert s.check_bvh() == 0
    s.close()
    specs = [dict(config=0, level=3, seed=11, width=64, height=48, spp=4, max_depth=5, guided=0),
             dict(config=3, level=3, seed=14, width=48, height=64, spp=3, max_depth=7, guided=0)]
    imgs = []
    for qn in (False, True):
        b = pathed.Session(16, 16)
        b.set_bvh_quantized(qn)
        b.load_batch(specs)
        b.render(0)
        b.render(0)
        imgs.append([b.batch_readback(i) for i in range(2)])
        b.close()
    for a, c in zip(*imgs):
        assert np.array_equal(a, c)

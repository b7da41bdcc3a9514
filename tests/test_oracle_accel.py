"""The oracle's parity accelerator against the oracle's own linear scan (World::hit,
src/world.cu:5-41). The accelerator exists so that parity runs on the 1.31M-triangle meshes
finish in seconds; it is trusted only because it returns the scan's answers bit for bit:
closest-hit primitive, material and t on seeded ray sets, and identical rendered pixels."""
import numpy as np
import pytest

import pathed
from _util import pixel_subset, seeded_rays

SMALL = [(0, None), (1, None), (2, 4), (3, 4)]


def _scene(cfg, level):
    s = pathed.Session(16, 16)
    s.load_config(cfg, level=level)
    sc = s.export_scene()
    s.close()
    return sc


@pytest.mark.parametrize("case", SMALL, ids=lambda c: f"cfg{c[0]}")
def test_accelerated_closest_hits_equal_the_scan(oracle_lib, case):
    sc = _scene(*case)
    o, d, tmin, tmax = seeded_rays(sc, 20000, seed=41)
    a = oracle_lib.trace(oracle_lib.scene(sc), o, d, tmin, tmax)
    b = oracle_lib.trace(oracle_lib.scene(sc, accel=True), o, d, tmin, tmax)
    for k in ("prim_type", "prim_id", "mat_id", "t"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("cfg", [2, 3])
def test_accelerated_closest_hits_on_the_full_mesh(oracle_lib, cfg):
    """1,310,720-triangle icosphere (configuration 3 adds the 2,002-triangle room)"""
    sc = _scene(cfg, None)
    assert sc["tri_vertices"].shape[0] >= 1310720
    o, d, tmin, tmax = seeded_rays(sc, 600, seed=42 + cfg)
    a = oracle_lib.trace(oracle_lib.scene(sc), o, d, tmin, tmax)
    b = oracle_lib.trace(oracle_lib.scene(sc, accel=True), o, d, tmin, tmax)
    assert (a["prim_type"] >= 0).mean() > 0.3
    for k in ("prim_type", "prim_id", "mat_id", "t"):
        assert np.array_equal(a[k], b[k]), k


@pytest.mark.parametrize("case", [(1, None), (3, 4)], ids=lambda c: f"cfg{c[0]}")
@pytest.mark.parametrize("trace_once", [True, False])
def test_accelerated_render_equals_the_scan(oracle_lib, case, trace_once):
    """shadow queries stop at their first occluder through the accelerator; the flag and so
    every pixel stay the scan's"""
    sc = _scene(*case)
    w, h = 48, 48
    pix = pixel_subset(w, h, 200, seed=2)
    depth = 8 if case[0] == 1 else 10
    outs = []
    for accel in (False, True):
        osc = oracle_lib.scene(sc, accel=accel)
        outs.append(oracle_lib.render(osc, sc["camera"], w, h, pix, 2, depth, nee=True, seed=77,
                                      trace_once=trace_once))
    assert np.array_equal(outs[0][0], outs[1][0])
    assert np.array_equal(outs[0][2], outs[1][2])  # query counts

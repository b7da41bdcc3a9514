"""The opt-in watertight triangle test (Woop, Benthin and Wald 2013) against the reference's
Triangle::hit (src/primitives/triangle.cu:7-48), which is not watertight.

Crack rays: from points inside the closed, consistently wound icosphere mesh towards its
vertices and edge midpoints. Every such ray leaves the star-shaped mesh through the point it
aims at, so a miss is a crack. The reference's arithmetic misses a large share of them at
vertices; the watertight test misses none. Elsewhere the two tests agree except for rays
that pass within rounding distance of an edge (they may pick the other triangle of the
edge, at the same t)."""
import numpy as np
import pytest

import pathed
from _util import seeded_rays

FLT_MAX = np.float32(3.4028234663852886e38)


def mesh_scene(level):
    s = pathed.Session(16, 16)
    s.load_config(2, level=level)
    sc = s.export_scene()
    s.close()
    return sc


def crack_rays(sc, n, seed):
    """rays from near the mesh centre through vertices (odd) and edge midpoints (even)"""
    tv = sc["tri_vertices"].reshape(-1, 3, 3)
    rng = np.random.default_rng(seed)
    ti = rng.integers(0, tv.shape[0], n)
    k = rng.integers(0, 3, n)
    a, b = tv[ti, k], tv[ti, (k + 1) % 3]
    p = np.where((np.arange(n) % 2 == 1)[:, None], a, (a + b) * np.float32(0.5)).astype(np.float32)
    o = (tv.reshape(-1, 3).mean(0) + rng.normal(size=(n, 3)) * 0.05).astype(np.float32)
    d = (p - o).astype(np.float32)
    return o, d, np.zeros(n, np.float32), np.full(n, FLT_MAX, np.float32)


def classify(ref, wt):
    """crack-misses (reference misses, watertight hits), ties (both hit the same distance
    within 1e-4 relative on different triangles), others"""
    r_hit, w_hit = ref["prim_type"] >= 0, wt["prim_type"] >= 0
    diff = (ref["prim_type"] != wt["prim_type"]) | (ref["prim_id"] != wt["prim_id"])
    crack = ~r_hit & w_hit
    tie = diff & r_hit & w_hit & (np.abs(ref["t"] - wt["t"]) <= 1e-4 * np.abs(wt["t"]))
    other = diff & ~crack & ~tie
    return int(crack.sum()), int(tie.sum()), int(other.sum())


def test_oracle_watertight_has_no_cracks(oracle_lib):
    sc = mesh_scene(5)
    o, d, tmin, tmax = crack_rays(sc, 20000, seed=3)
    ref = oracle_lib.trace(oracle_lib.scene(sc, accel=True), o, d, tmin, tmax)
    wt = oracle_lib.trace(oracle_lib.scene(sc, accel=True, watertight=True), o, d, tmin, tmax)
    crack, tie, other = classify(ref, wt)
    print(f"20,480-triangle mesh, 20,000 rays through vertices and edges: the reference's test misses "
          f"{crack} (crack-misses), {tie} ties, {other} other differences; the watertight test misses "
          f"{int((wt['prim_type'] < 0).sum())}")
    assert (wt["prim_type"] < 0).sum() == 0
    assert crack > 100  # the rays do probe the reference's cracks
    assert other == 0


@pytest.mark.parametrize("case", [(0, None), (1, None), (3, 4)], ids=lambda c: f"cfg{c[0]}")
def test_oracle_watertight_agrees_off_edges(oracle_lib, case):
    s = pathed.Session(16, 16)
    s.load_config(case[0], level=case[1])
    sc = s.export_scene()
    s.close()
    o, d, tmin, tmax = seeded_rays(sc, 20000, seed=8)
    ref = oracle_lib.trace(oracle_lib.scene(sc), o, d, tmin, tmax)
    wt = oracle_lib.trace(oracle_lib.scene(sc, watertight=True), o, d, tmin, tmax)
    crack, tie, other = classify(ref, wt)
    same = (ref["prim_id"] == wt["prim_id"]) & (ref["prim_type"] == wt["prim_type"])
    print(f"cfg{case[0]}: {(~same).sum()} of 20,000 seeded rays differ: {crack} crack-misses, {tie} ties, "
          f"{other} other")
    # the Cornell box's quads split along a diagonal: rays through it tie on the two halves
    assert other == 0 and crack <= 20 and same.mean() >= 0.99
    # spheres keep Sphere::hit's test, so their hits are bit-identical
    sph = (ref["prim_type"] == 1) | (wt["prim_type"] == 1)
    assert np.array_equal(ref["t"][sph & same], wt["t"][sph & same])


@pytest.mark.gpu
@pytest.mark.parametrize("case", [(0, None), (1, None), (2, 4), (3, 4)], ids=lambda c: f"cfg{c[0]}")
def test_gpu_watertight_bitexact_vs_oracle(oracle_lib, case):
    s = pathed.Session(16, 16)
    s.load_config(case[0], level=case[1])
    s.set_watertight(True)
    sc = s.export_scene()
    o, d, tmin, tmax = seeded_rays(sc, 20000, seed=9)
    g = s.trace_rays(o, d, tmin, tmax)
    r = oracle_lib.trace(oracle_lib.scene(sc, watertight=True), o, d, tmin, tmax)
    for k in ("prim_type", "prim_id", "mat_id", "t"):
        bad = np.nonzero(g[k] != r[k])[0]
        assert bad.size == 0, f"{k}: {bad.size} differ"
    s.close()


@pytest.mark.gpu
def test_gpu_crack_misses_of_the_reference_test(oracle_lib):
    """the full 1,310,720-triangle mesh: the GPU's default (reference) test against its
    watertight mode on crack rays, counted as crack-misses, ties and others"""
    sc = mesh_scene(8)
    o, d, tmin, tmax = crack_rays(sc, 50000, seed=4)
    s = pathed.Session(16, 16)
    s.load_config(2)
    ref = s.trace_rays(o, d, tmin, tmax)
    s.set_watertight(True)
    wt = s.trace_rays(o, d, tmin, tmax)
    s.set_watertight(False)
    again = s.trace_rays(o, d, tmin, tmax)
    s.close()
    crack, tie, other = classify(ref, wt)
    print(f"1,310,720-triangle mesh, 50,000 rays through vertices and edges: the reference's test misses "
          f"{crack} ({crack / 500:.2f}%, crack-misses), {tie} ties on the neighbouring triangle, {other} other "
          f"differences; the watertight test misses {int((wt['prim_type'] < 0).sum())}")
    assert (wt["prim_type"] < 0).sum() == 0 and other == 0 and crack > 0
    orc = oracle_lib.trace(oracle_lib.scene(sc, accel=True, watertight=True), o, d, tmin, tmax)
    for k in ("prim_type", "prim_id", "t"):
        assert np.array_equal(wt[k], orc[k]), k
    for k in ("prim_type", "prim_id", "t"):  # switching back restores the reference's test
        assert np.array_equal(again[k], ref[k]), k


@pytest.mark.gpu
def test_gpu_watertight_frames_same_stream(oracle_lib):
    """frames with the watertight test: closest hits and shadow rays through it, per pixel
    against the oracle in the same mode on the same random streams"""
    from _util import pixel_subset

    w = h = 64
    s = pathed.Session(w, h)
    s.load_config(0)
    s.set_watertight(True)
    s.render(8)
    img = s.readback().reshape(-1, 3).astype(np.float64)
    sc = s.export_scene()
    depth = s.counts().default_depth
    s.close()
    pix = pixel_subset(w, h, 1500, seed=6)
    mean, _, _ = oracle_lib.render(oracle_lib.scene(sc, watertight=True), sc["camera"], w, h, pix, 8, depth,
                                   nee=True, trace_once=True)
    close = np.all(np.abs(img[pix] - mean) <= 1e-3 * np.abs(mean) + 1e-5, axis=1).mean()
    assert close >= 0.99

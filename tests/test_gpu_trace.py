"""Closest-hit / any-hit parity of the sm_100a BVH traversal against the reference's
intersection code (World::hit, src/world.cu:5-41), through the C ABI.

The oracle's linear scan restates World::hit and is itself checked bit for bit against the
reference's own World::hit compiled for the CPU (test_oracle_ref.py). Here the GPU result
must equal it exactly: primitive type, primitive id, material id and the hit distance t.
"""
import numpy as np
import pytest

import pathed
from _util import FLT_MAX, seeded_rays

CONFIGS = [(0, None, 30000), (1, None, 30000), (2, 4, 12000), (3, 4, 12000)]


@pytest.fixture(scope="module", params=CONFIGS, ids=lambda c: f"cfg{c[0]}-lvl{c[1]}")
def loaded(request, oracle_lib):
    cfg, level, n = request.param
    s = pathed.Session(64, 64)
    s.load_config(cfg, level=level)
    sc = s.export_scene()
    yield s, sc, oracle_lib.scene(sc), n
    s.close()


def _compare(g, r):
    for k in ("prim_type", "prim_id", "mat_id", "t"):
        bad = np.nonzero(g[k] != r[k])[0]
        assert bad.size == 0, f"{k}: {bad.size} rays differ, first {bad[:5]}: gpu {g[k][bad[:5]]} oracle {r[k][bad[:5]]}"


@pytest.mark.gpu
@pytest.mark.parametrize("width", [2, 4, 8])
def test_closest_hit_bitexact(loaded, oracle_lib, width):
    s, sc, osc, n = loaded
    s.set_bvh(width, 4)
    o, d, tmin, tmax = seeded_rays(sc, n, seed=width)
    g = s.trace_rays(o, d, tmin, tmax)
    r = oracle_lib.trace(osc, o, d, tmin, tmax)
    assert (r["prim_type"] >= 0).sum() > n // 10
    _compare(g, r)


@pytest.mark.gpu
def test_closest_hit_leaf_sizes(loaded, oracle_lib):
    s, sc, osc, n = loaded
    o, d, tmin, tmax = seeded_rays(sc, n // 2, seed=11)
    r = oracle_lib.trace(osc, o, d, tmin, tmax)
    for leaf in (1, 8, 16):
        s.set_bvh(4, leaf)
        _compare(s.trace_rays(o, d, tmin, tmax), r)
    s.set_bvh(4, 4)


@pytest.mark.gpu
def test_bounded_queries(loaded, oracle_lib):
    """finite tmax (shadow-ray style) and tmin at the reference's epsilons"""
    s, sc, osc, n = loaded
    o, d, tmin, _ = seeded_rays(sc, n // 2, seed=5)
    rng = np.random.default_rng(5)
    tmax = rng.uniform(0.01, 5.0, o.shape[0]).astype(np.float32)
    r = oracle_lib.trace(osc, o, d, tmin, tmax)
    _compare(s.trace_rays(o, d, tmin, tmax), r)
    occ = s.occluded(o, d, tmin, tmax)
    assert np.array_equal(occ, (r["prim_type"] >= 0).astype(np.int32))


@pytest.mark.gpu
def test_device_pointer_entry(loaded, oracle_lib):
    torch = pytest.importorskip("torch")
    s, sc, osc, n = loaded
    o, d, tmin, tmax = seeded_rays(sc, 4096, seed=3)
    dev = {k: torch.from_numpy(v).cuda() for k, v in dict(o=o, d=d, tmin=tmin, tmax=tmax).items()}
    m = 4096
    out = {k: torch.empty(m, dtype=torch.int32, device="cuda") for k in ("pt", "pid", "mid")}
    t = torch.empty(m, dtype=torch.float32, device="cuda")
    torch.cuda.synchronize()
    rc = pathed.lib.pt_trace_rays_device(s._h, dev["o"].data_ptr(), dev["d"].data_ptr(), dev["tmin"].data_ptr(),
                                         dev["tmax"].data_ptr(), m, out["pt"].data_ptr(), out["pid"].data_ptr(),
                                         out["mid"].data_ptr(), t.data_ptr(), None)
    assert rc == 0, pathed.lib.pt_last_error(s._h)
    r = oracle_lib.trace(osc, o, d, tmin, tmax)
    assert np.array_equal(out["pid"].cpu().numpy(), r["prim_id"])
    assert np.array_equal(t.cpu().numpy(), r["t"])


@pytest.mark.gpu
def test_hit_test_matches_camera_ray(oracle_lib):
    s = pathed.Session(128, 96)
    s.load_config(0)
    sc = s.export_scene()
    osc = oracle_lib.scene(sc)
    rng = np.random.default_rng(2)
    import oracle as orc

    for _ in range(40):
        x, y = int(rng.integers(0, 128)), int(rng.integers(0, 96))
        mat = s.hit_test(x, y)
        ray = np.zeros(6, np.float32)
        oracle_lib.lib.oracle_camera_ray(orc._f(sc["camera"]).ctypes.data, 128, 96, y, x, 0.5, 0.5, ray.ctypes.data)
        r = oracle_lib.trace(osc, ray[:3][None], ray[3:][None], 0.0, FLT_MAX)
        assert mat == r["mat_id"][0]
    assert s.hit_test(-1, 5) == -1  # outside the image: no thread matches (hit_test.cu:35)
    s.close()


@pytest.mark.gpu
def test_full_size_mesh_bitexact(oracle_lib):
    """1,310,720-triangle displaced icosphere (configuration 2 at full size), fewer rays"""
    s = pathed.Session(64, 64)
    s.load_config(2)
    sc = s.export_scene()
    assert sc["counts"].num_triangles == 1310720
    osc = oracle_lib.scene(sc)
    o, d, tmin, tmax = seeded_rays(sc, 1500, seed=9)
    _compare(s.trace_rays(o, d, tmin, tmax), oracle_lib.trace(osc, o, d, tmin, tmax))
    s.close()

"""Pin the oracle (oracle/oracle.cpp) against the reference itself (CPU).

tests/golden/reference_vectors.npz holds outputs of the reference's own code, compiled for
the host from the reference sources (tests/golden/make_golden.py), on the inputs of the
reference's distribution tests (test/test_distribution.cu) and on seeded unit inputs. The
oracle must reproduce every value bit for bit; the distribution results must also meet the
reference tests' own expected values (Catch2 Approx tolerance, 100 float epsilons).
"""
import os

import numpy as np
import pytest

import oracle as orc

HERE = os.path.dirname(os.path.abspath(__file__))
G = np.load(os.path.join(HERE, "golden", "reference_vectors.npz"))
APPROX = 100 * np.finfo(np.float32).eps  # Catch2 Approx default epsilon


def approx(a, b):
    return np.all(np.abs(np.asarray(a, np.float64) - b) <= APPROX * (np.abs(b) + 1.0))


def same(a, b):
    return np.array_equal(np.asarray(a), np.asarray(b), equal_nan=True)


@pytest.fixture(scope="module")
def O():
    return orc.Oracle()


def test_distribution_pmf_and_mass(O):  # test_distribution.cu:42-123
    pmf, total, _, _ = orc.dist1d(O, G["dist1d_values"], G["dist1d_xis"][:1])
    assert approx(pmf, G["dist1d_expect_pmf"]) and approx(total, G["dist1d_expect_total"])
    assert same(pmf, G["dist1d_ref_pmf"]) and total == G["dist1d_ref_total"]
    pmf, _, _, _ = orc.dist1d(O, np.zeros(2, np.float32), np.zeros(0, np.float32))
    assert np.all(pmf == 0.0) and same(pmf, G["dist1d_empty_ref_pmf"])  # :73-95


def test_distribution_sampling(O):  # test_distribution.cu:125-197
    _, _, idx, spmf = orc.dist1d(O, G["dist1d_s_values"], G["dist1d_xis"])
    assert np.array_equal(idx, G["dist1d_expect_idx"]) and approx(spmf, G["dist1d_expect_spmf"])
    assert np.array_equal(idx, G["dist1d_ref_idx"]) and same(spmf, G["dist1d_ref_spmf"])


def test_distribution_xi_one_and_random(O):
    pmf, total, idx, spmf = orc.dist1d(O, G["rd_values"], G["rd_xis"])
    assert same(pmf, G["rd_ref_pmf"]) and total == G["rd_ref_total"]
    assert np.array_equal(idx, G["rd_ref_idx"]) and same(spmf, G["rd_ref_spmf"])
    assert idx[-3] >= 0  # xi == 1 lands on the first index whose CDF is 1 (distribution.h:36-43)


def test_distribution2d(O):  # test_distribution.cu:263-380
    pmf, sx, sy, spmf = orc.dist2d(O, G["dist2d_values"], 2, 4, G["dist2d_xis"])
    assert approx(pmf.ravel(), G["dist2d_expect_pmf"]) and same(pmf.ravel(), G["dist2d_ref_pmf"])
    idx = np.stack([sx, sy], 1)
    assert np.array_equal(idx, G["dist2d_expect_idx"]) and np.array_equal(idx, G["dist2d_ref_idx"])
    assert approx(spmf, G["dist2d_expect_spmf"]) and same(spmf, G["dist2d_ref_spmf"])


def test_phitheta_pdf(O):  # test_distribution.cu:415-494
    pc, pd = orc.phitheta_pdf(O, G["dist2d_values"], 2, 4, G["pt_canon"], G["pt_dirs"])
    assert same(pc, G["pt_ref_pdf_canon"]) and same(pd, G["pt_ref_pdf_dir"])
    assert abs(pc.mean() - 1.0) < 1e-5  # canonical pdf integrates to 1 (:448-453)
    assert abs(np.mean(pd * 4 * np.pi) - 1.0) < 5e-2  # spherical pdf integrates to 1 (:488-493)


@pytest.mark.parametrize("t", [0, 1, 2, 3], ids=["lambert", "mirror", "glass", "beckmann"])
def test_bsdf_sample_and_eval(O, t):
    wo, wi, xi, alb = G["bsdf_wo"], G["bsdf_wi"], G["bsdf_xi"], G["bsdf_albedo"]
    smp = np.zeros((len(wo), 8), np.float32)
    ev = np.zeros((len(wo), 4), np.float32)
    for k in range(len(wo)):
        O.lib.oracle_bsdf_sample(t, alb.ctypes.data, 1.5, 0.3, wo[k].ctypes.data, float(xi[k, 0]), float(xi[k, 1]),
                                 smp[k].ctypes.data)
        O.lib.oracle_bsdf_eval(t, alb.ctypes.data, 1.5, 0.3, wo[k].ctypes.data, wi[k].ctypes.data, ev[k].ctypes.data)
    assert same(smp, G[f"bsdf{t}_sample"])
    assert same(ev, G[f"bsdf{t}_eval"])


def _scene_from_golden(O, cfg):
    import pathed

    s = pathed.Session(64, 48)
    s.load_config(cfg)
    sc = s.export_scene()
    s.close()
    return sc, O.scene(sc)


@pytest.mark.parametrize("cfg", [0, 1])
def test_closest_hit(O, cfg):
    sc, osc = _scene_from_golden(O, cfg)
    r = O.trace(osc, G[f"s{cfg}_o"], G[f"s{cfg}_d"], G[f"s{cfg}_tmin"], G[f"s{cfg}_tmax"])
    for k in ("prim_type", "prim_id", "mat_id", "t"):
        assert same(r[k], G[f"s{cfg}_hit_{k}"]), k


@pytest.mark.parametrize("cfg", [0, 1])
def test_emitter_samples(O, cfg):
    sc, osc = _scene_from_golden(O, cfg)
    pts, lx = G[f"s{cfg}_lpts"], G[f"s{cfg}_lxi"]
    out = np.zeros((len(pts), 11), np.float32)
    for k in range(len(pts)):
        O.lib.oracle_light_sample(osc.h, pts[k].ctypes.data, float(lx[k, 0]), float(lx[k, 1]), float(lx[k, 2]),
                                  out[k].ctypes.data)
    assert same(out, G[f"s{cfg}_light"])


@pytest.mark.parametrize("cfg", [0, 1])
def test_camera_rays(O, cfg):
    cam, rc, cx = G[f"s{cfg}_cam"], G[f"s{cfg}_cam_rc"], G[f"s{cfg}_cam_xi"]
    out = np.zeros((len(rc), 6), np.float32)
    for k in range(len(rc)):
        O.lib.oracle_camera_ray(cam.ctypes.data, 64, 48, int(rc[k, 0]), int(rc[k, 1]), float(cx[k, 0]),
                                float(cx[k, 1]), out[k].ctypes.data)
    assert same(out, G[f"s{cfg}_cam_ray"])


@pytest.mark.parametrize("cfg", [0, 1])
def test_normals_gbuffer(O, cfg):
    """the normals renderer's image (g_buffer.cu:27-57): pixel-centre rays, (n + 1) / 2"""
    sc, osc = _scene_from_golden(O, cfg)
    img = O.normals(osc, G[f"s{cfg}_cam"], 64, 48)
    assert same(img, G[f"s{cfg}_normals"])
    assert (img == 0).all(-1).sum() < img.shape[0] * img.shape[1]  # not all misses


def test_environment_samples(O):
    env = G["env_map"]
    sc = {"tri_vertices": np.zeros((1, 9), np.float32), "tri_normals": np.zeros((1, 9), np.float32),
          "tri_materials": np.zeros(1, np.int32), "spheres": np.zeros((0, 4), np.float32),
          "sphere_materials": np.zeros(0, np.int32), "material_types": np.zeros(1, np.int32),
          "material_albedo": np.zeros((1, 3), np.float32), "material_emit": np.zeros((1, 3), np.float32),
          "material_ior": np.ones(1, np.float32), "material_alpha": np.ones(1, np.float32), "env_rgba": env}
    osc = O.scene(sc)
    ex = G["env_xi"]
    out = np.zeros((len(ex), 7), np.float32)
    for k in range(len(ex)):
        O.lib.oracle_env_sample(osc.h, float(ex[k, 0]), float(ex[k, 1]), out[k].ctypes.data)
    assert same(out, G["env_sample"])


def test_fixture_matches_reference_build(ref_lib):
    """Where the reference CPU build is present, it still produces the committed fixture."""
    pmf, total, idx, spmf = orc.dist1d(ref_lib, G["rd_values"], G["rd_xis"])
    assert same(pmf, G["rd_ref_pmf"]) and np.array_equal(idx, G["rd_ref_idx"])

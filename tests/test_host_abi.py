"""Host-side checks of the C ABI (no GPU): every declared symbol is exported, scene
generation and the BVH builder behave, and invalid input is rejected with an error code
instead of a crash or an exit (the reference exits through gpuAssert,
include/macro_helper.h:10-19)."""
import os
import re
import subprocess

import numpy as np
import pytest

import pathed

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def test_header_symbols_exported():
    hdr = open(os.path.join(ROOT, "include", "pathed.h")).read()
    declared = set(re.findall(r"^(?:int|const char\*)\s+(pt_\w+)\(", hdr, flags=re.M))
    assert declared, "no declarations found"
    out = subprocess.run(["nm", "-D", "--defined-only", pathed.LIB_PATH], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (pt_\w+)", out))
    assert declared <= exported, f"missing: {sorted(declared - exported)}"
    assert declared == set(pathed.EXPORTED)


def test_library_built_for_sm100a():
    out = subprocess.run(["cuobjdump", "--list-elf", pathed.LIB_PATH], capture_output=True, text=True).stdout
    assert "sm_100a" in out


@pytest.mark.parametrize("cfg,ntri,nsph,nlights", [(0, 36, 0, 2), (1, 2, 68, 4)])
def test_config_contents(cfg, ntri, nsph, nlights):
    s = pathed.Session(32, 32)
    s.load_config(cfg)
    c = s.counts()
    assert (c.num_triangles, c.num_spheres, c.num_lights) == (ntri, nsph, nlights)
    assert s.check_bvh() == 0
    sc = s.export_scene()
    if cfg == 0:
        # emitter quad of area 0.25 with radiance 15, facing down
        lt = sc["light_indices"]
        tv = sc["tri_vertices"][lt].reshape(-1, 3, 3)
        area = 0.5 * np.linalg.norm(np.cross(tv[:, 1] - tv[:, 0], tv[:, 2] - tv[:, 0]), axis=1).sum()
        assert abs(area - 0.25) < 1e-5
        assert np.allclose(sc["material_emit"][sc["tri_materials"][lt]], 15.0)
        n = np.cross(tv[:, 1] - tv[:, 0], tv[:, 2] - tv[:, 0])
        assert np.all(n[:, 1] < 0)
    if cfg == 1:
        types = sc["material_types"][sc["sphere_materials"][:64]]
        # 40% Beckmann: F0 0.04 (the reference's dielectric Fresnel) or a metallic RGB F0
        beck = (types == pathed.MICROFACET) | (types == pathed.METAL)
        assert beck.sum() == 26 and (types == pathed.MIRROR).sum() == 13
        metal = sc["material_types"] == pathed.METAL
        assert 6 <= metal.sum() <= 20
        f0 = sc["material_albedo"][metal]
        assert np.all((f0 > 0.3) & (f0 <= 1.0))
        alpha = sc["material_alpha"][sc["sphere_materials"][:64]][beck]
        assert alpha.min() >= 0.05 and alpha.max() <= 0.5
        assert (types == pathed.GLASS).sum() == 13 and (types == pathed.LAMBERTIAN).sum() == 12
        r = sc["spheres"][:64, 3]
        assert r.min() >= 0.2 and r.max() <= 1.0
    s.close()


def test_configs_are_seeded_and_deterministic():
    a = pathed.Session(8, 8)
    b = pathed.Session(8, 8)
    a.load_config(1, seed=5)
    b.load_config(1, seed=5)
    assert np.array_equal(a.export_scene()["spheres"], b.export_scene()["spheres"])
    b.load_config(1, seed=6)
    assert not np.array_equal(a.export_scene()["spheres"], b.export_scene()["spheres"])


@pytest.mark.parametrize("level,ntri", [(3, 20 * 4 ** 3 + 0), (5, 20 * 4 ** 5)])
def test_icosphere_levels(level, ntri):
    s = pathed.Session(8, 8)
    s.load_config(2, level=level)
    c = s.counts()
    assert c.num_triangles == ntri and c.env_width == 2048 and c.env_height == 1024
    s.load_config(3, level=level)
    assert s.counts().num_triangles == ntri + 2002


@pytest.mark.parametrize("width", [2, 4, 8])
@pytest.mark.parametrize("leaf", [1, 4, 16])
def test_bvh_structure(width, leaf):
    s = pathed.Session(8, 8)
    s.load_config(3, level=4)
    s.set_bvh(width, leaf)
    c = s.counts()
    assert c.bvh_width == width and c.bvh_max_leaf <= leaf
    assert s.check_bvh() == 0


def test_invalid_input_is_an_error_not_a_crash():
    with pytest.raises(pathed.PathedError):
        pathed.Session(0, 10)
    s = pathed.Session(16, 16)
    with pytest.raises(pathed.PathedError):
        s.load_config(9)
    with pytest.raises(pathed.PathedError):
        s.render(4)  # no scene
    s.load_config(0)
    with pytest.raises(pathed.PathedError):
        s.set_bvh(3, 4)
    with pytest.raises(pathed.PathedError):
        s.set_max_depth(-1)
    with pytest.raises(pathed.PathedError):
        s.set_material(99, 0)
    with pytest.raises(pathed.PathedError):
        s.set_camera((0, 1, 0), (0, 0, 0), (0, 1, 0), 0.5)  # look direction equals up
    with pytest.raises(pathed.PathedError):
        s.set_launch(block_extend=48)
    with pytest.raises(pathed.PathedError) as e:
        s.load_arrays(tri_vertices=np.array([[0, 0, 0, 1, 0, 0, 0, np.nan, 0]]), tri_materials=[0],
                      material_types=[0], material_albedo=[[1, 1, 1]], material_emit=[[0, 0, 0]])
    assert "non-finite" in str(e.value)
    with pytest.raises(pathed.PathedError):
        s.load_arrays(tri_vertices=np.zeros((1, 9)), tri_materials=[3], material_types=[0])
    s.close()


def test_launch_config_host_state():
    """launch options are host state: ray sorting defaults off, 0 keeps a field, bad modes fail"""
    s = pathed.Session(16, 16)
    s.load_config(0)
    cfg = s.get_launch()
    assert cfg["sort_rays"] == 2 and cfg["use_graph"] == 1 and cfg["sort_materials"] == 3
    s.set_launch(sort_rays=1)
    assert s.get_launch()["sort_rays"] == 1
    s.set_launch(block_extend=256)  # other fields 0: unchanged
    assert s.get_launch()["sort_rays"] == 1 and s.get_launch()["block_extend"] == 256
    for bad in (-1, 3):
        with pytest.raises(pathed.PathedError):
            s.set_launch(sort_rays=bad)
    s.set_launch(sort_rays=2)
    assert s.get_launch()["sort_rays"] == 2
    assert cfg["refill_idle"] == 16
    s.set_launch(refill_idle=32)
    assert s.get_launch()["refill_idle"] == 32
    for bad in (-1, 33):
        with pytest.raises(pathed.PathedError):
            s.set_launch(refill_idle=bad)
    assert cfg["speculate"] == 2
    for code in (1, 3, 4, 2):  # both stages, closest hit only, shadow only, off
        s.set_launch(speculate=code)
        assert s.get_launch()["speculate"] == code
    with pytest.raises(pathed.PathedError):
        s.set_launch(speculate=5)
    # concurrent shadow stage and fused camera rays on by default, node-order shadow traversal
    assert cfg["overlap_shadow"] == 1 and cfg["fuse_camera"] == 1 and cfg["shadow_order"] == 2
    for field in ("overlap_shadow", "shadow_order", "fuse_camera", "split_shade"):
        start = s.get_launch()[field]
        for code in (1, 2):
            s.set_launch(**{field: code})
            assert s.get_launch()[field] == code
        s.set_launch(**{field: start})
        for bad in (-1, 5):
            with pytest.raises(pathed.PathedError) as e:
                s.set_launch(**{field: bad})
            assert e.value.code == pathed.PT_ERR_ARG
    s.close()


def test_load_arrays_roundtrip():
    s = pathed.Session(16, 16)
    s.load_config(1)
    sc = s.export_scene()
    t = pathed.Session(16, 16)
    t.load_arrays(sc["tri_vertices"], sc["tri_normals"], sc["tri_materials"], sc["spheres"], sc["sphere_materials"],
                  sc["material_types"], sc["material_albedo"], sc["material_emit"], sc["material_ior"],
                  sc["material_alpha"])
    sc2 = t.export_scene()
    for k in ("tri_vertices", "spheres", "material_types", "light_indices", "light_types"):
        assert np.array_equal(sc[k], sc2[k]), k
    # without normals: each vertex takes the triangle's normalised geometric normal
    t.load_arrays(tri_vertices=[[0, 0, 0, 1, 0, 0, 0, 1, 0]], tri_materials=[0], material_types=[0],
                  material_albedo=[[1, 1, 1]], material_emit=[[0, 0, 0]])
    assert np.allclose(t.export_scene()["tri_normals"].reshape(3, 3), [[0, 0, 1]] * 3)
    s.close()
    t.close()


def test_device_calls_fail_cleanly_without_gpu():
    torch = pytest.importorskip("torch")
    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    s = pathed.Session(16, 16)
    s.load_config(0)
    with pytest.raises(pathed.PathedError) as e:
        s.render(1)
    assert e.value.code == pathed.PT_ERR_CUDA
    with pytest.raises(pathed.PathedError):  # nothing rendered: no image to copy out
        s.readback_async(np.empty((16, 16, 3), np.float32))
    assert s.readback_wait() is None  # nothing pending: returns at once
    s.close()

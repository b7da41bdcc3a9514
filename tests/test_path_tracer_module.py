"""The pybind11 module `path_tracer`: the reference GUI's binding surface
(bindings/path_tracer_bindings.cu:10-87) over libpathed, headless."""
import numpy as np
import pytest

import path_tracer as ptm
import pathed

# every name the reference module exports, by class
REFERENCE_SURFACE = {
    "RenderSession": ["init", "renderAsync", "pollRender", "hitTest", "getWidth", "getHeight", "getSceneModel"],
    "SceneModel": ["getRendererType", "setRendererType", "setColor", "getColor", "setEmit", "getEmit", "getIOR",
                   "setIOR", "getAlpha", "setAlpha", "getMaterialID", "getMaterialType", "setMaterialType",
                   "setLightPosition", "getLightPosition", "getCameraOrigin", "setCameraOrigin", "getCameraTarget",
                   "setCameraTarget", "getCameraUp", "setCameraUp", "getMaxDepth", "setMaxDepth",
                   "getNextEventEstimation", "setNextEventEstimation", "zoomCamera", "getSpp"],
    "Vec3": ["x", "y", "z", "r", "g", "b"],
    "RenderState": ["isRendering", "pbo"],
    "MaterialIndex": ["materialType", "index"],
}


def test_module_mirrors_reference_surface():
    for cls, names in REFERENCE_SURFACE.items():
        c = getattr(ptm, cls)
        missing = [n for n in names if not hasattr(c, n)]
        assert not missing, (cls, missing)
    # enum values as in materials/types.h:5-11 and scene_model.h:15-19
    assert [int(v) for v in (ptm.Lambertian, ptm.Mirror, ptm.Glass, ptm.Microfacet)] == [0, 1, 2, 3]
    assert {ptm.RendererType.CUDA, ptm.RendererType.Optix, ptm.RendererType.Normals}


def test_scene_model_host_state():
    s = ptm.RenderSession(64, 48)
    assert (s.getWidth(), s.getHeight()) == (64, 48)
    m = s.getSceneModel()
    # no material selected yet (scene_model.cu:56-140)
    assert m.getMaterialID() == -1
    c = m.getColor()
    assert (c.r(), c.g(), c.b()) == (0.0, 0.0, 0.0)
    assert m.getIOR() == -1.0 and m.getAlpha() == -1.0
    assert m.getMaterialType() == getattr(ptm.MaterialType, "None")  # a keyword in Python
    assert m.getRendererType() == ptm.RendererType.CUDA
    assert m.getLightPosition() == pytest.approx(-0.6)
    # configuration 0's camera and defaults
    ref = pathed.Session(64, 48)
    ref.load_config(0)
    cam = ref.export_scene()["camera"]
    o = m.getCameraOrigin()
    assert (o.x(), o.y(), o.z()) == tuple(float(v) for v in cam[0:3])
    counts = ref.counts()
    assert m.getMaxDepth() == counts.default_depth
    assert m.getNextEventEstimation() == bool(counts.default_nee)
    ref.close()
    with pytest.raises(RuntimeError):
        m.setRendererType(ptm.RendererType.Optix)
    m.setRendererType(ptm.RendererType.Normals)  # the G-buffer (g_buffer.cu)
    assert m.getRendererType() == ptm.RendererType.Normals
    m.setRendererType(ptm.RendererType.CUDA)
    assert m.getRendererType() == ptm.RendererType.CUDA
    with pytest.raises(RuntimeError):
        s.renderAsync()  # init() first
    # scene selection beyond the reference's hard-coded scene 0
    s.load_scene(1)
    assert m.getMaxDepth() == 8 and m.getMaterialID() == -1
    ex = ref_arrays()
    s.load_scene_arrays(**ex)
    o = m.getCameraOrigin()
    assert np.isfinite([o.x(), o.y(), o.z()]).all()
    with pytest.raises(ValueError):
        bad = dict(ex)
        bad["tri_materials"] = bad["tri_materials"][:-1]
        s.load_scene_arrays(**bad)


def ref_arrays():
    r = pathed.Session(32, 32)
    r.load_config(0)
    e = r.export_scene()
    r.close()
    return dict(tri_vertices=e["tri_vertices"], tri_normals=e["tri_normals"], tri_materials=e["tri_materials"],
                spheres=e["spheres"], sphere_materials=e["sphere_materials"], material_types=e["material_types"],
                material_albedo=e["material_albedo"], material_emit=e["material_emit"],
                material_ior=e["material_ior"], material_alpha=e["material_alpha"], env_rgba=None)


def _frame(s):
    st = s.renderAsync()
    assert st.isRendering
    while s.pollRender().isRendering:
        pass


@pytest.mark.gpu
def test_render_loop_and_spp_budget():
    s = ptm.RenderSession(128, 128)
    st = s.init()
    assert not st.isRendering and st.pbo == 0
    m = s.getSceneModel()
    _frame(s)
    assert m.getSpp() == 1  # one sample after a reset (spp_optimizer.cpp:19-23)
    _frame(s)
    second = m.getSpp() - 1
    assert second >= 1  # then as many as fit 80 ms at the measured rate
    for _ in range(3):
        _frame(s)
    img = s.getRadianceBuffer()
    assert img.shape == (128, 128, 3) and np.isfinite(img).all() and img.mean() > 0


@pytest.mark.gpu
def test_hit_test_and_material_edits():
    s = ptm.RenderSession(96, 96)
    s.init()
    _frame(s)
    _frame(s)
    m = s.getSceneModel()
    s.hitTest(48, 48)
    mid = m.getMaterialID()
    ref = pathed.Session(96, 96)
    ref.load_config(0)
    assert mid == ref.hit_test(48, 48)
    alb = ref.export_scene()["material_albedo"].reshape(-1, 3)[mid]
    c = m.getColor()
    assert np.allclose([c.r(), c.g(), c.b()], alb)
    ref.close()
    m.setColor(0.1, 0.2, 0.3)
    c = m.getColor()
    assert np.allclose([c.r(), c.g(), c.b()], [0.1, 0.2, 0.3])
    _frame(s)
    assert m.getSpp() == 1  # the edit restarted accumulation
    m.setMaterialType(ptm.MaterialType.Mirror)
    assert m.getMaterialType() == ptm.MaterialType.Mirror
    m.setMaxDepth(2)
    assert m.getMaxDepth() == 2
    m.setNextEventEstimation(False)
    assert not m.getNextEventEstimation()
    o0, t0 = m.getCameraOrigin(), m.getCameraTarget()
    m.zoomCamera(0.5)
    o1 = m.getCameraOrigin()
    d = np.array([t0.x() - o0.x(), t0.y() - o0.y(), t0.z() - o0.z()])
    d /= np.linalg.norm(d)
    assert np.allclose([o1.x() - o0.x(), o1.y() - o0.y(), o1.z() - o0.z()], 0.5 * d, atol=1e-6)
    _frame(s)
    assert np.isfinite(s.getRadianceBuffer()).all()
    rgba = s.readback_rgba8()
    assert rgba.shape == (96, 96, 4) and (rgba[..., 3] == 255).all()

"""Normals renderer (the reference's GBuffer with BufferType::Normals, src/renderers/g_buffer.cu):
each frame traces one pixel-centre camera ray per pixel and writes (normal + 1) / 2 of the
closest hit, black on a miss, into the running mean as a 1-spp pass.

The oracle's image is pinned against the reference's own code (tests/test_oracle_golden.py);
here the CUDA path is compared with it bit for bit: the camera ray, the closest hit and the
normal are each computed with every FP32 operation rounded in the reference's order."""
import os

import numpy as np
import pytest

import oracle as orc
import pathed

HERE = os.path.dirname(os.path.abspath(__file__))


def _session(config, level, w, h, width=4, leaf=4):
    s = pathed.Session(w, h)
    s.load_config(config, level=level)
    s.set_bvh(width, leaf)
    return s


def test_renderer_switch_host_rules():
    s = _session(0, None, 32, 32)
    with pytest.raises(pathed.PathedError):
        s.set_renderer(pathed.RENDERER_OPTIX)
    s.set_renderer(pathed.RENDERER_NORMALS)
    with pytest.raises(pathed.PathedError):  # batches render with the path tracer only
        s.load_batch([dict(config=0, level=-1, seed=1, width=32, height=32, spp=1, max_depth=3, guided=0)])
    s.set_renderer(pathed.RENDERER_CUDA)
    s.load_batch([dict(config=0, level=-1, seed=1, width=32, height=32, spp=1, max_depth=3, guided=0)])
    with pytest.raises(pathed.PathedError):
        s.set_renderer(pathed.RENDERER_NORMALS)
    s.close()


def _compare(img, ref):
    miss_g = (img == 0).all(-1)
    miss_o = (ref == 0).all(-1)
    assert miss_o.mean() < 1.0
    err = float(np.abs(img - ref).max())
    assert np.array_equal(miss_g, miss_o), f"{int((miss_g != miss_o).sum())} pixels hit on one side only"
    assert np.array_equal(img, ref), f"max |GPU - oracle| {err:.3e} on {int((img != ref).any(-1).sum())} pixels"
    return err


@pytest.mark.gpu
@pytest.mark.parametrize("cfg", [0, 1])
def test_normals_match_golden_image(cfg):
    """64 x 48, the committed image of the reference's own G-buffer arithmetic"""
    g = np.load(os.path.join(HERE, "golden", "reference_vectors.npz"))
    s = _session(cfg, None, 64, 48)
    assert np.array_equal(s.export_scene()["camera"], g[f"s{cfg}_cam"])
    s.set_renderer(pathed.RENDERER_NORMALS)
    s.render(1)
    _compare(s.readback(), g[f"s{cfg}_normals"])
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("config,level,width,leaf", [(2, 3, 8, 4), (3, 3, 2, 2), (1, 3, 4, 1)])
def test_normals_match_oracle_on_meshes(config, level, width, leaf):
    w, h = 96, 72
    s = _session(config, level, w, h, width, leaf)
    sc = s.export_scene()
    O = orc.Oracle()
    ref = O.normals(O.scene(sc), sc["camera"], w, h)
    s.set_renderer(pathed.RENDERER_NORMALS)
    s.render(1)
    err = _compare(s.readback(), ref)
    print(f"config {config} level {level}: max |GPU - oracle| {err:.2e}")
    s.close()


@pytest.mark.gpu
def test_normals_frames_accumulate_one_sample_each():
    s = _session(3, 3, 128, 128)
    s.set_renderer(pathed.RENDERER_NORMALS)
    s.render(16)  # the G-buffer renders one sample whatever is asked
    first = s.readback().copy()
    assert s.spp() == 1
    s.render(4)
    s.render(1)
    assert s.spp() == 3
    assert float(np.abs(s.readback() - first).max()) <= 1e-6  # the mean of identical passes
    st = s.stats()
    assert st["rays_camera"] == 128 * 128 and st["rays_shadow"] == 0
    # back to the path tracer: accumulation restarts
    s.set_renderer(pathed.RENDERER_CUDA)
    s.render(4)
    assert s.spp() == 4
    img = s.readback()
    assert np.isfinite(img).all() and not np.array_equal(img, first)
    s.close()


@pytest.mark.gpu
def test_module_normals_renderer():
    import path_tracer as ptm

    w, h = 80, 64
    rs = ptm.RenderSession(w, h)
    rs.init()
    m = rs.getSceneModel()
    m.setRendererType(ptm.RendererType.Normals)
    assert m.getRendererType() == ptm.RendererType.Normals
    for k in range(3):
        rs.renderAsync()
        while rs.pollRender().isRendering:
            pass
        assert m.getSpp() == k + 1
    ref = _session(0, None, w, h)
    ref.set_renderer(pathed.RENDERER_NORMALS)
    ref.render(1)
    assert float(np.abs(rs.getRadianceBuffer() - ref.readback()).max()) <= 1e-6
    ref.close()

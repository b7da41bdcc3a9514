"""Configuration 1's metallic-RGB Beckmann spheres ("F0 0.04 or a metallic RGB"). The reference
has no such material (its Microfacet uses a dielectric Fresnel of fixed eta 1.5,
include/materials/microfacet.h:111), so the material is judged against the oracle only:
  * the oracle's metal BSDF equals its Beckmann D and G (the reference's, pinned by the
    golden vectors) times Schlick's Fresnel of RGB F0, restated here in FP64;
  * the GPU renders a scene of metal spheres on the oracle's random streams, per pixel."""
import numpy as np
import pytest

import pathed
from _util import pixel_subset


def _dielectric(c, eta_i=1.0, eta_t=1.5):
    """fresnel.h's dielectric reflectance, FP64"""
    s_i = np.sqrt(max(0.0, 1 - c * c))
    s_t = eta_i / eta_t * s_i
    if s_t >= 1:
        return 1.0
    c_t = np.sqrt(max(0.0, 1 - s_t * s_t))
    rpar = (eta_t * c - eta_i * c_t) / (eta_t * c + eta_i * c_t)
    rper = (eta_i * c - eta_t * c_t) / (eta_i * c + eta_t * c_t)
    return (rpar * rpar + rper * rper) / 2


def test_oracle_metal_is_beckmann_with_schlick_fresnel(oracle_lib):
    rng = np.random.default_rng(5)
    f0 = np.array([0.955, 0.638, 0.538], np.float32)
    alpha = 0.3
    n = 0
    for _ in range(400):
        wo = rng.normal(size=3)
        wi = rng.normal(size=3)
        wo[2], wi[2] = abs(wo[2]), abs(wi[2])
        wo = (wo / np.linalg.norm(wo)).astype(np.float32)
        wi = (wi / np.linalg.norm(wi)).astype(np.float32)
        m = np.zeros(4, np.float32)
        d = np.zeros(4, np.float32)
        oracle_lib.lib.oracle_bsdf_eval(pathed.METAL, f0.ctypes.data, 1.5, alpha, wo.ctypes.data, wi.ctypes.data,
                                        m.ctypes.data)
        oracle_lib.lib.oracle_bsdf_eval(pathed.MICROFACET, f0.ctypes.data, 1.5, alpha, wo.ctypes.data,
                                        wi.ctypes.data, d.ctypes.data)
        wh = (wo.astype(np.float64) + wi) / np.linalg.norm(wo.astype(np.float64) + wi)
        c = min(1.0, max(0.0, float(wi @ wh)))
        fd = _dielectric(c)
        if d[0] <= 0 or fd <= 0:
            continue
        dg = d[0] / fd  # D G / (4 cos_i cos_o) of the reference's Beckmann
        expect = dg * (f0 + (1 - f0) * (1 - c) ** 5)
        assert np.allclose(m[:3], expect, rtol=2e-4, atol=1e-7)
        assert m[3] == d[3]  # same sampling density
        n += 1
    assert n > 300


@pytest.mark.gpu
def test_metal_spheres_same_stream(oracle_lib):
    """configuration 1 with every Beckmann sphere metallic (gold, silver, copper and
    aluminium F0, their own roughness), GPU against the oracle on the same random streams"""
    w = h = 96
    s = pathed.Session(w, h)
    s.load_config(1)
    sc = s.export_scene()
    beck = np.nonzero((sc["material_types"] == pathed.MICROFACET) | (sc["material_types"] == pathed.METAL))[0]
    f0s = [(1.0, 0.766, 0.336), (0.972, 0.960, 0.915), (0.955, 0.638, 0.538), (0.913, 0.922, 0.924)]
    for k, i in enumerate(beck):
        s.set_material(int(i), pathed.METAL)
        s.set_material(int(i), pathed.METAL, albedo=f0s[k % 4], alpha=float(sc["material_alpha"][i]))
    sc = s.export_scene()
    assert (sc["material_types"] == pathed.METAL).sum() == len(beck) == 26
    s.render(8)
    img = s.readback().reshape(-1, 3).astype(np.float64)
    depth = s.counts().default_depth
    s.close()
    pix = pixel_subset(w, h, 2000, seed=12)
    mean, _, _ = oracle_lib.render(oracle_lib.scene(sc), sc["camera"], w, h, pix, 8, depth, nee=True,
                                   trace_once=True)
    tight = np.all(np.abs(img[pix] - mean) <= 1e-3 * np.abs(mean) + 1e-5, axis=1).mean()
    assert tight >= 0.9
    assert abs(img[pix].mean() - mean.mean()) <= 0.02 * abs(mean.mean()) + 1e-4

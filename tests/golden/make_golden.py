"""Generate tests/golden/reference_vectors.npz from the reference's own code.

Runs the reference sources compiled for the host CPU (oracle/_ref/libref_cpu.so, built by
`make -C oracle ref` from the reference tree) on:
  * the inputs of the reference's distribution tests (test/test_distribution.cu:42-494),
    whose expected values are stored beside the outputs;
  * seeded unit inputs for Triangle/Sphere/World::hit, the four BSDFs (sample, f, pdf), the
    emitter sampler, Camera::generateRay and the environment light.

    python tests/golden/make_golden.py

The fixture lets the CPU test suite pin the oracle on machines without the reference tree.
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "gpu-pathed_b200"), os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import oracle as orc  # noqa: E402
import pathed  # noqa: E402
from _util import seeded_rays  # noqa: E402

OUT = os.path.join(HERE, "reference_vectors.npz")

# ---- inputs and expected values of test/test_distribution.cu ------------------------------
DIST1D_VALUES = np.array([1, 1, 0, 3], np.float32)                 # :43-48
DIST1D_PMF = np.array([0.2, 0.2, 0.0, 0.6], np.float32)             # :67-70
DIST1D_TOTAL = 5.0                                                  # :122
DIST1D_EMPTY = np.array([0, 0], np.float32)                         # :74
DIST1D_S_VALUES = np.array([1, 1, 0, 3, 0], np.float32)             # :126-132
ETA = np.float32(1e-5)
DIST1D_XIS = np.array([0.0, 0.1 - ETA, 0.2 - ETA, 0.3 - ETA, 0.4 - ETA], np.float32)  # :135-144 (first 5 used)
DIST1D_IDX = np.array([0, 0, 0, 1, 1], np.int32)                    # :146-148
DIST1D_SPMF = np.array([0.2, 0.2, 0.2, 0.2, 0.2], np.float32)       # :150-152
DIST2D_VALUES = np.array([1, 4, 1, 0, 0, 0, 3, 1], np.float32)      # :267-272 (2 x 4)
DIST2D_PMF = np.array([0.1, 0.4, 0.1, 0.0, 0.0, 0.0, 0.3, 0.1], np.float32)  # :274-279
DIST2D_XIS = np.array([0.0, 0.2 - ETA, 0.1 - ETA, 0.3 - ETA, 0.51, 1.0, 0.7 - ETA, 0.75 - ETA,
                       0.7 - ETA, 0.76], np.float32)                 # :315-321
DIST2D_IDX = np.array([[0, 0], [1, 0], [0, 1], [0, 3], [1, 3]], np.int32)  # :323-329 (x, y)
DIST2D_SPMF = np.array([0.1, 0.4, 0.1, 0.3, 0.1], np.float32)       # :331-333


def small_env(seed=3, w=16, h=8):
    rng = np.random.default_rng(seed)
    env = rng.lognormal(0, 1, (h, w, 4)).astype(np.float32)
    env[..., 3] = 1.0
    env[2, 5, :3] = 200.0   # a bright texel
    env[6, :, :3] = 0.0     # an empty row
    return env


def unit_dirs(rng, n):
    v = rng.normal(0, 1, (n, 3))
    return (v / np.linalg.norm(v, axis=1, keepdims=True)).astype(np.float32)


def main():
    ref = orc.RefCPU()
    L = ref.lib
    rng = np.random.default_rng(2024)
    out = {}
    # distribution tests
    pmf, total, idx, spmf = orc.dist1d(ref, DIST1D_VALUES, DIST1D_XIS[:1])
    out.update(dist1d_values=DIST1D_VALUES, dist1d_ref_pmf=pmf, dist1d_ref_total=np.float32(total),
               dist1d_expect_pmf=DIST1D_PMF, dist1d_expect_total=np.float32(DIST1D_TOTAL))
    pmf, total, _, _ = orc.dist1d(ref, DIST1D_EMPTY, np.zeros(0, np.float32))
    out.update(dist1d_empty_ref_pmf=pmf)
    pmf, total, idx, spmf = orc.dist1d(ref, DIST1D_S_VALUES, DIST1D_XIS)
    out.update(dist1d_s_values=DIST1D_S_VALUES, dist1d_xis=DIST1D_XIS, dist1d_ref_idx=idx, dist1d_ref_spmf=spmf,
               dist1d_expect_idx=DIST1D_IDX, dist1d_expect_spmf=DIST1D_SPMF)
    pmf2, sx, sy, sp2 = orc.dist2d(ref, DIST2D_VALUES, 2, 4, DIST2D_XIS)
    out.update(dist2d_values=DIST2D_VALUES, dist2d_xis=DIST2D_XIS, dist2d_ref_pmf=pmf2.ravel(),
               dist2d_ref_idx=np.stack([sx, sy], 1), dist2d_ref_spmf=sp2, dist2d_expect_pmf=DIST2D_PMF,
               dist2d_expect_idx=DIST2D_IDX, dist2d_expect_spmf=DIST2D_SPMF)
    # phi-theta pdf: canonical grid (x8 multiplier, :427-453) and seeded sphere directions
    m = 8
    gx, gy = np.meshgrid((np.arange(2 * m) + 0.5) / (2 * m), (np.arange(4 * m) + 0.5) / (4 * m))
    canon = np.stack([gx.ravel(), gy.ravel()], 1).astype(np.float32)
    dirs = unit_dirs(rng, 4000)
    pc, pd = orc.phitheta_pdf(ref, DIST2D_VALUES, 2, 4, canon, dirs)
    out.update(pt_canon=canon, pt_dirs=dirs, pt_ref_pdf_canon=pc, pt_ref_pdf_dir=pd)
    # random 1-D distributions with random variates, incl. xi = 1 and zero runs
    vals = rng.uniform(0, 1, 257).astype(np.float32)
    vals[rng.random(257) < 0.3] = 0.0
    vals[-20:] = 0.0
    xis = np.concatenate([rng.uniform(0, 1, 500), [1.0, 2 ** -24, 0.5]]).astype(np.float32)
    pmf, total, idx, spmf = orc.dist1d(ref, vals, xis)
    out.update(rd_values=vals, rd_xis=xis, rd_ref_pmf=pmf, rd_ref_total=np.float32(total), rd_ref_idx=idx,
               rd_ref_spmf=spmf)
    # BSDFs: sample (with explicit variates) and f/pdf, per type
    n = 400
    wo = unit_dirs(rng, n)
    wo[: n // 4, 2] = -np.abs(wo[: n // 4, 2])  # some below the surface
    wi = unit_dirs(rng, n)
    xi = rng.uniform(0, 1, (n, 2)).astype(np.float32)
    xi[0] = [1.0, 1.0]
    albedo = np.array([0.7, 0.5, 0.3], np.float32)
    for t in range(4):
        smp = np.zeros((n, 8), np.float32)
        ev = np.zeros((n, 4), np.float32)
        for k in range(n):
            L.ref_bsdf_sample(t, albedo.ctypes.data, 1.5, 0.3, wo[k].ctypes.data, float(xi[k, 0]), float(xi[k, 1]),
                              smp[k].ctypes.data)
            L.ref_bsdf_eval(t, albedo.ctypes.data, 1.5, 0.3, wo[k].ctypes.data, wi[k].ctypes.data, ev[k].ctypes.data)
        out[f"bsdf{t}_sample"] = smp
        out[f"bsdf{t}_eval"] = ev
    out.update(bsdf_wo=wo, bsdf_wi=wi, bsdf_xi=xi, bsdf_albedo=albedo)
    # scenes: closest hit, emitter samples, camera rays, environment samples
    for cfg, level in ((0, None), (1, None)):
        s = pathed.Session(64, 48)
        s.load_config(cfg, level=level)
        sc = s.export_scene()
        s.close()
        rs = ref.scene(sc)
        o, d, tmin, tmax = seeded_rays(sc, 3000, seed=cfg + 10)
        hit = ref.trace(rs, o, d, tmin, tmax)
        out.update({f"s{cfg}_o": o, f"s{cfg}_d": d, f"s{cfg}_tmin": tmin, f"s{cfg}_tmax": tmax})
        for k, v in hit.items():
            out[f"s{cfg}_hit_{k}"] = v
        pts = (o[:500] + 0.5 * d[:500]).astype(np.float32)
        lx = rng.uniform(0, 1, (500, 3)).astype(np.float32)
        ls = np.zeros((500, 11), np.float32)
        for k in range(500):
            L.ref_light_sample(rs.h, pts[k].ctypes.data, float(lx[k, 0]), float(lx[k, 1]), float(lx[k, 2]),
                               ls[k].ctypes.data)
        out.update({f"s{cfg}_lpts": pts, f"s{cfg}_lxi": lx, f"s{cfg}_light": ls})
        cam = orc._f(sc["camera"])
        rc = rng.integers(0, [48, 64], (300, 2)).astype(np.int32)
        cx = rng.uniform(0, 1, (300, 2)).astype(np.float32)
        cr = np.zeros((300, 6), np.float32)
        for k in range(300):
            L.ref_camera_ray(cam.ctypes.data, 64, 48, int(rc[k, 0]), int(rc[k, 1]), float(cx[k, 0]), float(cx[k, 1]),
                             cr[k].ctypes.data)
        out.update({f"s{cfg}_cam": cam, f"s{cfg}_cam_rc": rc, f"s{cfg}_cam_xi": cx, f"s{cfg}_cam_ray": cr})
        # the normals G-buffer image (g_buffer.cu:27-57) at 64 x 48
        out[f"s{cfg}_normals"] = ref.normals(rs, cam, 64, 48)
    # environment light on a small synthetic map (sample, pdf, emit)
    env = small_env()
    scene_env = {"tri_vertices": np.zeros((1, 9), np.float32), "tri_normals": np.zeros((1, 9), np.float32),
                 "tri_materials": np.zeros(1, np.int32), "spheres": np.zeros((0, 4), np.float32),
                 "sphere_materials": np.zeros(0, np.int32), "material_types": np.zeros(1, np.int32),
                 "material_albedo": np.zeros((1, 3), np.float32), "material_emit": np.zeros((1, 3), np.float32),
                 "material_ior": np.ones(1, np.float32), "material_alpha": np.ones(1, np.float32), "env_rgba": env}
    rs = ref.scene(scene_env)
    ex = rng.uniform(0, 1, (1000, 2)).astype(np.float32)
    ex[0] = [1.0, 1.0]
    es = np.zeros((1000, 7), np.float32)
    for k in range(1000):
        L.ref_env_sample(rs.h, float(ex[k, 0]), float(ex[k, 1]), es[k].ctypes.data)
    out.update(env_map=env, env_xi=ex, env_sample=es)
    np.savez_compressed(OUT, **out)
    print("wrote", OUT, os.path.getsize(OUT), "bytes")


if __name__ == "__main__":
    main()

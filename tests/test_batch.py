"""Batched frames (configuration 4): many scenes in one session, every wavefront stage one
launch over all scenes' rays. A batched scene's paths draw the same random streams and run
the same arithmetic as the scene rendered alone, so its image must be bit-identical."""
import numpy as np
import pytest

import pathed


def test_batch_draw_matches_configuration():
    a = pathed.batch_generate(0x5EED, 48)
    b = pathed.batch_generate(0x5EED, 48)
    assert a == b  # seeded
    assert pathed.batch_generate(7, 48) != a
    assert {d["config"] for d in a} == {0, 1, 2, 3}
    for d in a:
        assert 3 <= d["level"] <= 8  # 1,280 .. 1,310,720 mesh triangles (log-uniform 1k-2M)
        assert d["width"] == d["height"] and 256 <= d["width"] <= 1024 and d["width"] % 64 == 0
        assert d["spp"] in (4, 8, 16, 32, 64)
        assert 4 <= d["max_depth"] <= 10
    guided = sum(d["guided"] for d in a)
    assert 12 <= guided <= 36  # about half


SMALL = [
    dict(config=0, level=3, seed=11, width=96, height=64, spp=4, max_depth=5, guided=0),
    dict(config=1, level=-1, seed=12, width=64, height=64, spp=8, max_depth=6, guided=0),
    dict(config=2, level=4, seed=13, width=80, height=48, spp=2, max_depth=4, guided=0),
    dict(config=3, level=3, seed=14, width=64, height=96, spp=3, max_depth=7, guided=0),
]


def test_batch_merge_host_side():
    s = pathed.Session(16, 16)
    s.load_batch(SMALL)
    tot_tri = tot_px = tot_paths = 0
    for i, d in enumerate(SMALL):
        info = s.batch_info(i)
        ref = pathed.Session(16, 16)
        ref.load_config(d["config"], seed=d["seed"], level=d["level"] if d["level"] >= 0 else None)
        c = ref.counts()
        ref.close()
        assert (info["num_triangles"], info["num_spheres"], info["num_lights"]) == \
            (c.num_triangles, c.num_spheres, c.num_lights)
        assert info["first_pixel"] == tot_px and info["first_path"] == tot_paths
        tot_tri += c.num_triangles
        tot_px += d["width"] * d["height"]
        tot_paths += d["width"] * d["height"] * d["spp"]
    assert s.counts().num_triangles == tot_tri
    # single-scene queries are refused for a batch
    with pytest.raises(pathed.PathedError):
        s.hit_test(0, 0)
    with pytest.raises(pathed.PathedError):
        s.set_material(0, 0, (1, 1, 1), (0, 0, 0), 1.5, 0.1)
    bad = dict(SMALL[0], spp=0)
    with pytest.raises(pathed.PathedError):
        s.load_batch([bad])
    s.close()


def _alone(d, frames):
    r = pathed.Session(d["width"], d["height"])
    r.load_config(d["config"], seed=d["seed"], level=d["level"] if d["level"] >= 0 else None)
    r.set_max_depth(d["max_depth"])
    for _ in range(frames):
        r.render(d["spp"])
    img = r.readback()
    st = r.stats()
    r.close()
    return img, st


@pytest.mark.gpu
@pytest.mark.parametrize("wave_paths", [0, 20000])
def test_batched_images_equal_scenes_rendered_alone(wave_paths):
    """bit-identical per scene; wave_paths 20000 splits scenes across many waves"""
    s = pathed.Session(16, 16)
    s.load_batch(SMALL)
    if wave_paths:
        s.set_launch(wave_paths=wave_paths)
    frames = 2
    for _ in range(frames):
        s.render(0)
    st = s.stats()
    assert st["rays_camera"] == sum(d["width"] * d["height"] * d["spp"] for d in SMALL)
    rays = 0
    for i, d in enumerate(SMALL):
        img = s.batch_readback(i)
        ref, rst = _alone(d, frames)
        assert s.batch_info(i)["spp_accumulated"] == frames * d["spp"]
        assert np.array_equal(img, ref), (i, float(np.abs(img - ref).max()))
        rays += rst["rays_extend"] + rst["rays_shadow"]
    assert st["rays_extend"] + st["rays_shadow"] == rays
    s.close()


@pytest.mark.gpu
def test_batch_reset_and_graph_replay():
    s = pathed.Session(16, 16)
    s.load_batch(SMALL[:2])
    s.render(0)
    s.render(0)
    a = s.batch_readback(1)
    s.reset()
    s.render(0)
    s.render(0)
    b = s.batch_readback(1)
    assert np.array_equal(a, b)  # same seeds after a reset
    assert s.batch_info(0)["spp_accumulated"] == 2 * SMALL[0]["spp"]
    s.close()


@pytest.mark.gpu
def test_guided_batch_one_network_per_guided_scene():
    specs = [dict(config=3, level=3, seed=21, width=64, height=64, spp=4, max_depth=8, guided=1),
             dict(config=0, level=-1, seed=22, width=64, height=64, spp=4, max_depth=5, guided=0),
             dict(config=2, level=3, seed=23, width=64, height=48, spp=4, max_depth=5, guided=1)]
    frames, skip = 32, 8
    s = pathed.Session(16, 16)
    s.load_batch(specs)
    s.set_guiding(True)
    means = []
    for k in range(frames):
        s.render(0)
        if k >= skip:
            means.append(s.batch_readback(0, pass_only=True).mean())
    info = s.guide_info()
    assert info["mode"] == 2 and info["steps"] > 0 and info["samples"] > 0
    # the unguided scene's paths are untouched by guiding (consistent MIS is on for the batch)
    ref = pathed.Session(64, 64)
    ref.load_config(0, seed=22)
    ref.set_max_depth(5)
    ref.set_consistent_mis(True)
    for _ in range(frames):
        ref.render(4)
    assert np.array_equal(s.batch_readback(1), ref.readback())
    ref.close()
    s.close()
    # the guided scene converges to its plain image: frame means within 4.5 standard errors
    plain = pathed.Session(64, 64)
    plain.load_config(3, seed=21, level=3)
    plain.set_max_depth(8)
    plain.set_consistent_mis(True)
    pm = []
    for _ in range(frames - skip):
        plain.render(4)
        pm.append(plain.readback(pass_only=True).mean())
    plain.close()
    m0, e0 = np.mean(pm), np.std(pm, ddof=1) / np.sqrt(len(pm))
    m1, e1 = np.mean(means), np.std(means, ddof=1) / np.sqrt(len(means))
    print(f"slit room in a guided batch: {m1:.6f} +- {e1:.6f}, alone plain {m0:.6f} +- {e0:.6f}")
    assert abs(m0 - m1) <= 4.5 * np.hypot(e0, e1)


@pytest.mark.gpu
def test_autotuner_on_a_batch(tmp_path):
    """the autotuner runs on batched frames too (BVH width and ray sorting fixed, wave size
    tuned), changes scheduling only, and caches its choice under the batch's own key"""
    cache = str(tmp_path / "tune.jsonl")
    s = pathed.Session(16, 16)
    s.load_batch(SMALL)
    s.set_seed(3)
    s.render(0)
    base = [s.batch_readback(k).copy() for k in range(len(SMALL))]
    r = s.autotune(1, cache)
    assert r["trials"] > 0 and r["from_cache"] == 0 and r["bvh_width"] == s.counts().bvh_width
    assert r["wave_paths"] > 0 and r["best_ms"] <= r["default_ms"] * 1.05
    s.render(0)  # tuning restarts accumulation: this is the first frame again
    for k in range(len(SMALL)):
        assert np.allclose(s.batch_readback(k), base[k], rtol=1e-5, atol=1e-6)
    t = pathed.Session(16, 16)
    t.load_batch(SMALL)
    r2 = t.autotune(1, cache)
    assert r2["from_cache"] == 1 and r2["wave_paths"] == r["wave_paths"] and r2["block"] == r["block"]
    u = pathed.Session(16, 16)
    u.load_batch(SMALL[:3])  # another draw: its own key, so it is measured
    assert u.autotune(1, cache)["from_cache"] == 0
    for x in (s, t, u):
        x.close()


@pytest.mark.gpu
def test_wave_size_does_not_change_images():
    """the autotuner's wave size splits a frame into more waves: same paths, same images"""
    out = []
    for wave in (1 << 25, 5000):
        s = pathed.Session(64, 48)
        s.load_config(1)
        s.set_launch(wave_paths=wave)
        s.render(8)
        out.append(s.readback().copy())
        s.close()
    assert np.allclose(out[0], out[1], rtol=1e-5, atol=1e-6)

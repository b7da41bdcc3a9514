"""Learned path guiding: the network kernels against the FP64 CPU oracle, unbiasedness of the
guided estimator, and what the trained guide gains over plain BSDF + NEE sampling.

CPU part: the oracle's analytic gradient of the loss -sum w log q(wi|x) / sum w is checked
against central finite differences (FP64), so that it can serve as the reference of the GPU
training kernel.
"""
import numpy as np
import pytest

import pathed

NP = pathed.GUIDE_PARAMS


def bf16_round(a):
    a = np.asarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    u = (u + 0x7FFF + ((u >> 16) & 1)) & 0xFFFF0000
    return u.astype(np.uint32).view(np.float32)


def random_params(seed=0, scale=1.0):
    rng = np.random.default_rng(seed)
    p = np.zeros(NP, np.float32)
    sizes = [(0, 80 * 64, 80), (5120 + 64, 64 * 64, 64), (9280 + 64, 64 * 64, 64), (13440 + 64, 64 * 40, 64)]
    for off, cnt, fan in sizes:
        p[off:off + cnt] = rng.normal(0, np.sqrt(2.0 / fan) * scale, cnt)
    p[5120:5184] = rng.normal(0, 0.1, 64)
    p[9280:9344] = rng.normal(0, 0.1, 64)
    p[13440:13504] = rng.normal(0, 0.1, 64)
    p[16064:] = rng.normal(0, 0.5, 40)
    return bf16_round(p)


def random_batch(n, seed=1):
    rng = np.random.default_rng(seed)
    x = rng.normal(0, 1, (n, 80)).astype(np.float32)
    x[:, 78:] = 0
    wi = rng.normal(0, 1, (n, 3))
    wi /= np.linalg.norm(wi, axis=1, keepdims=True)
    w = rng.exponential(1.0, n).astype(np.float32)
    w[rng.random(n) < 0.2] = 0
    return x, wi.astype(np.float32), w


def test_oracle_gradient_matches_finite_differences(oracle_lib):
    p = random_params(3, scale=0.5).astype(np.float64)
    x, wi, w = random_batch(24, seed=4)
    _, g = oracle_lib.guide_grad(p.astype(np.float32), x, wi, w)
    rng = np.random.default_rng(5)
    idx = np.concatenate([rng.choice(5120, 25, replace=False), 5120 + rng.choice(64, 5, replace=False),
                          9344 + rng.choice(4096, 20, replace=False), 13504 + rng.choice(2560, 30, replace=False),
                          16064 + np.arange(40)])
    h = 1e-6
    for i in idx:
        pp = p.copy(); pp[i] += h
        pm = p.copy(); pm[i] -= h
        fd = (oracle_lib.guide_loss_exact(pp, x, wi, w) - oracle_lib.guide_loss_exact(pm, x, wi, w)) / (2 * h)
        assert abs(fd - g[i]) <= 1e-5 + 1e-4 * abs(fd), (i, fd, g[i])


@pytest.mark.gpu
def test_inference_kernel_matches_oracle(oracle_lib):
    s = pathed.Session(8, 8)
    p = random_params(7)
    s.set_guide_params(p)
    x, _, _ = random_batch(1000, seed=8)
    raw = s.guide_forward(x).astype(np.float64)
    ref = oracle_lib.guide_forward(p, x, quant=True)  # BF16 operands, FP64 accumulation
    err = np.abs(raw - ref)
    scale = np.abs(ref).max()
    # FP32 accumulation and BF16 re-rounding of activations near rounding boundaries
    assert np.percentile(err, 99) <= 2e-2 * scale
    assert np.mean(err) <= 2e-3 * scale
    s.close()


@pytest.mark.gpu
def test_training_gradients_match_oracle(oracle_lib):
    s = pathed.Session(8, 8)
    p = random_params(9)
    s.set_guide_params(p)
    x, wi, w = random_batch(3000, seed=10)
    g = s.guide_gradients(x, wi, w).astype(np.float64)
    _, ref = oracle_lib.guide_grad(p, x, wi, w)
    rel = np.linalg.norm(g - ref) / np.linalg.norm(ref)
    cos = g @ ref / (np.linalg.norm(g) * np.linalg.norm(ref))
    assert rel <= 1e-3 and cos >= 0.999999, (rel, cos)
    s.close()


def _slit_room(w, h):
    s = pathed.Session(w, h)
    s.load_config(3, level=3)
    return s


@pytest.mark.gpu
def test_guided_estimator_is_unbiased():
    """guided frames converge to the plain (consistent-MIS) image: image mean within 4 SE"""
    w = h = 48
    frames, spp = 24, 16
    means = {}
    for guided in (False, True):
        s = _slit_room(w, h)
        s.set_consistent_mis(True)
        if guided:
            s.set_guiding(True)
            s.set_guide_options(steps_per_frame=4, warmup_steps=8)
        vals = []
        for k in range(frames):
            s.render(spp)
            if not guided or k >= 4:  # guided: frames after the guide is in use
                vals.append(s.readback(pass_only=True).mean())
        if guided:
            assert s.guide_info()["mode"] == 2
        means[guided] = (np.mean(vals), np.std(vals, ddof=1) / np.sqrt(len(vals)))
        s.close()
    (m0, e0), (m1, e1) = means[False], means[True]
    print(f"plain {m0:.6f} +- {e0:.6f}  guided {m1:.6f} +- {e1:.6f}")
    assert abs(m0 - m1) <= 4 * np.hypot(e0, e1)


@pytest.mark.gpu
def test_trained_guide_reduces_error():
    """hard lighting (environment seen through a slit): at equal samples, the trained guide's
    relMSE against a converged plain render is lower than plain BSDF + NEE sampling's"""
    w = h = 48
    ref = _slit_room(w, h)
    ref.set_consistent_mis(True)
    for _ in range(16):
        ref.render(256)
    img_ref = ref.readback().astype(np.float64)
    ref.close()

    def relmse(img):
        return float(np.mean((img - img_ref) ** 2 / (img_ref ** 2 + 1e-2)))

    plain = _slit_room(w, h)
    plain.set_consistent_mis(True)
    plain.set_seed(77)
    for _ in range(8):
        plain.render(16)
    e_plain = relmse(plain.readback().astype(np.float64))
    plain.close()

    g = _slit_room(w, h)
    g.set_guiding(True)
    g.set_guide_options(steps_per_frame=8, warmup_steps=16)
    for _ in range(12):  # training frames (discarded)
        g.render(16)
    g.reset()
    g.set_seed(77)
    for _ in range(8):
        g.render(16)
    e_guided = relmse(g.readback().astype(np.float64))
    info = g.guide_info()
    g.close()
    print(f"relMSE at 128 spp: plain {e_plain:.5f} guided {e_guided:.5f} (steps {info['steps']}, "
          f"samples {info['samples']})")
    assert e_guided < e_plain

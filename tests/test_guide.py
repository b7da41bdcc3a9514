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
@pytest.mark.parametrize("tc", [False, True], ids=["mma.sync", "tcgen05"])
def test_inference_kernel_matches_oracle(oracle_lib, tc):
    s = pathed.Session(8, 8)
    s.set_guide_inference(tc)
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
def test_tensor_memory_inference_equals_mma_sync():
    """both inference paths round the same operands: outputs agree to FP32 accumulation order"""
    s = pathed.Session(8, 8)
    s.set_guide_params(random_params(11))
    x, _, _ = random_batch(5000, seed=12)  # 40 tiles of 128 (one partial)
    a = s.guide_forward(x)
    s.set_guide_inference(True)
    b = s.guide_forward(x)
    s.close()
    scale = np.abs(a).max()
    assert np.percentile(np.abs(a - b), 99.9) <= 1e-2 * scale
    assert np.mean(np.abs(a - b)) <= 1e-4 * scale


def _compare(g, ref):
    rel = np.linalg.norm(g - ref) / np.linalg.norm(ref)
    cos = g @ ref / (np.linalg.norm(g) * np.linalg.norm(ref))
    return rel, cos


def test_bf16_operand_rounding_is_a_small_perturbation(oracle_lib):
    """the oracle's BF16 emulation of the training kernel stays close to exact FP64 training"""
    p = random_params(9)
    x, wi, w = random_batch(500, seed=10)
    _, exact = oracle_lib.guide_grad(p, x, wi, w)
    _, quant = oracle_lib.guide_grad(p, x, wi, w, quant=True)
    rel, cos = _compare(quant, exact)
    assert rel <= 3e-2 and cos >= 0.999, (rel, cos)


@pytest.mark.gpu
@pytest.mark.parametrize("tc", [False, True], ids=["mma.sync", "tcgen05"])
@pytest.mark.parametrize("n", [3000, 40000])
def test_training_gradients_match_oracle(oracle_lib, n, tc):
    """tensor-core training kernels (BF16 operands, FP32 accumulation; mma.sync, or tcgen05
    with the weight-gradient accumulators in tensor memory) against the FP64 oracle that
    rounds the same operands to BF16; n = 40000 gives blocks several sample tiles"""
    s = pathed.Session(8, 8)
    s.set_guide_training(tc)
    p = random_params(9)
    s.set_guide_params(p)
    x, wi, w = random_batch(n, seed=10)
    g = s.guide_gradients(x, wi, w).astype(np.float64)
    _, ref_q = oracle_lib.guide_grad(p, x, wi, w, quant=True)
    _, ref = oracle_lib.guide_grad(p, x, wi, w)
    rel_q, cos_q = _compare(g, ref_q)
    rel, cos = _compare(g, ref)
    print(f"n {n}: vs BF16-emulating oracle rel {rel_q:.2e} cos {cos_q:.8f}; vs exact rel {rel:.2e}")
    # FP32 accumulation order and rare BF16 rounding-boundary flips are all that differ
    assert rel_q <= 2e-3 and cos_q >= 0.99999, (rel_q, cos_q)
    assert rel <= 3e-2 and cos >= 0.999, (rel, cos)
    # every parameter block is trained: per-block agreement
    for lo, hi in [(0, 5120), (5120, 5184), (5184, 9280), (9280, 9344), (9344, 13440), (13440, 13504),
                   (13504, 16064), (16064, 16104)]:
        r, _ = _compare(g[lo:hi], ref_q[lo:hi])
        assert r <= 1e-2, (lo, hi, r)
    s.close()


def _slit_room(w, h):
    s = pathed.Session(w, h)
    s.load_config(3, level=3)
    return s


@pytest.mark.gpu
@pytest.mark.parametrize("tc,fraction", [(False, None), (True, None), (False, 0.3)],
                         ids=["mma.sync", "tcgen05", "mma.sync-fraction0.3"])
def test_guided_estimator_is_unbiased(tc, fraction):
    """guided frames converge to the plain (consistent-MIS) image: image mean within 4 SE, at
    the default guide fraction and at another one"""
    w = h = 48
    frames, spp = 24, 16
    means = {}
    for guided in (False, True):
        s = _slit_room(w, h)
        s.set_consistent_mis(True)
        if guided:
            s.set_guide_inference(tc)
            if fraction is not None:
                s.set_guide_fraction(fraction)
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
    """hard lighting (environment seen through a slit): after online training, the guided
    render's relMSE against a converged plain render is clearly below plain BSDF + NEE
    sampling's at the same sample count"""
    w = h = 128
    ref = _slit_room(w, h)
    ref.set_consistent_mis(True)
    ref.set_seed(1234)
    for _ in range(16):
        ref.render(512)
    img_ref = ref.readback().astype(np.float64)
    ref.close()

    def relmse(img):
        return float(np.mean((img - img_ref) ** 2 / (img_ref ** 2 + 1e-2)))

    plain = _slit_room(w, h)
    plain.set_consistent_mis(True)
    plain.set_seed(77)
    for _ in range(16):
        plain.render(4)
    e_plain = relmse(plain.readback().astype(np.float64))
    plain.close()

    g = _slit_room(w, h)
    g.set_guiding(True)
    g.set_guide_options(steps_per_frame=8, batch=1 << 16, warmup_steps=4)
    for _ in range(96):  # online training frames (discarded)
        g.render(4)
    g.reset()
    g.set_seed(77)
    for _ in range(16):
        g.render(4)
    e_guided = relmse(g.readback().astype(np.float64))
    info = g.guide_info()
    g.close()
    print(f"relMSE at 64 spp: plain {e_plain:.6f} guided {e_guided:.6f} (ratio {e_plain / e_guided:.2f}; "
          f"steps {info['steps']}, samples {info['samples']}, loss {info['loss']:.3f})")
    assert info["mode"] == 2
    assert e_guided < 0.8 * e_plain


def test_guide_fraction_range():
    s = pathed.Session(16, 16)
    for bad in (0.0, 1.0, -0.5, float("nan")):
        with pytest.raises(pathed.PathedError):
            s.set_guide_fraction(bad)
    s.set_guide_fraction(0.9)
    s.close()


@pytest.mark.gpu
def test_tcgen05_training_in_frames():
    """guided frames whose online training runs on tcgen05: the loss falls and the image stays
    finite; the same frames trained on mma.sync reach a loss of the same size"""
    losses = {}
    for tc in (True, False):
        s = _slit_room(48, 48)
        s.set_seed(21)
        s.set_guide_training(tc)
        s.set_guiding(True)
        s.set_guide_options(steps_per_frame=4, warmup_steps=8)
        trace = []
        for f in range(32):
            s.render(4)
            trace.append(s.guide_info()["loss"])
        early, late = float(np.mean(trace[2:6])), float(np.mean(trace[-6:]))
        losses[tc] = (early, late, s.guide_info()["steps"])
        assert np.all(np.isfinite(s.readback())) and np.all(np.isfinite(trace))
        s.close()
    print("loss early / late / steps:", losses)
    e_tc, l_tc, steps = losses[True]
    assert steps >= 96 and l_tc < e_tc
    assert abs(l_tc - losses[False][1]) <= 0.5 * abs(losses[False][1]) + 0.5

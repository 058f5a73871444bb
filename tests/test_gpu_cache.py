"""GPU parity of the radiance cache (tcgen05 MLP, cached path tracer).

Bars (written next to each assertion):
  * inference: the FP16/FP32 numpy model (tests/rc_reference.py) to
    accumulation-order noise (a hidden activation whose FP16 rounding flips
    moves an output by ~1e-3 of the output scale); within 2e-2 relative
    (RMS) of the unrounded FP32 network
  * training step: loss to 1e-4 relative; gradient within 1e-2 relative
    (RMS over all weights) of the FP16 model and 5e-2 of the unrounded FP32
    gradient; the Adam update exactly as written from the reported gradient
  * cached path tracer with a constant cache: per pixel within 1e-4 relative
    of the oracle's cached estimator for >= 99% of pixels; with a zero cache
    bit-identical to the plain path tracer truncated at the cache depth; the
    per-path tail kernel bit-identical to the wavefront stages
  * online training on the Cornell box (800 Adam steps): the median loss of
    the last 10 frames is at most half that of the first 10,
    and per channel the cached image's mean radiance recovers at least half
    of what ending paths at the cache depth loses against a converged plain
    render (the cache is a biased estimator; this bounds its bias)
"""
import os
import tempfile

import numpy as np
import pytest
import torch

import cupbr_b200 as cb
from cupbr_b200 import scenes
from cupbr_b200.cache import RadianceCache
from oracle.bridge import CheckerScene

import rc_reference as R

pytestmark = pytest.mark.gpu

_built = {}


def cornell():
    if "c" not in _built:
        _built["c"] = scenes.cornell_box().build()
    return _built["c"]


def dev(a):
    return torch.as_tensor(np.ascontiguousarray(a, np.float32), device="cuda")


def rel_rms(a, b):
    return float(np.sqrt(np.mean((a - b) ** 2)) / max(np.sqrt(np.mean(b ** 2)), 1e-30))


def plain(sc, w, h, depth, frames):
    r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    r.set_output_size(w, h)
    r.register_scene(sc)
    r.set_method(cb.RenderingMethod.PATHTRACER)
    r.set_max_trace_depth(depth)
    r.set_russian_roulette(False)
    r.render_frames(cb.Camera(w, h), frames)
    return r.get_output_image().numpy()


def cached(c, sc, w, h, frames, depth, train=False, frame0=0):
    img = torch.zeros((h, w, 3), device="cuda")
    c.render(sc, cb.Camera(w, h), w, h, frame0, frames, depth, img.data_ptr(), train=train)
    torch.cuda.synchronize()
    return img.cpu().numpy()


def test_infer_matches_model():
    sc = cornell()
    c = RadianceCache(sc)
    lo, inv = c.bounds()
    p = R.init_params(1)
    c.set_params(p)
    n = 1000  # ragged last tile
    recs = R.random_records(n, lo, lo + 1.0 / inv, seed=2, targets=False)
    out = torch.zeros((n, 4), device="cuda")
    c.infer(dev(recs).data_ptr(), n, out.data_ptr())
    torch.cuda.synchronize()
    y = out.cpu().numpy()[:, :3]
    assert c.counters()[0] == 0
    ym, _ = R.forward(p, R.encode(recs, lo, inv))
    assert np.abs(y - ym).max() <= 2e-3 * np.abs(ym).max() + 1e-6       # FP16 model, accumulation order
    ye, _ = R.forward(p, R.encode(recs, lo, inv, rounded=False), rounded=False)
    assert rel_rms(y, ye) <= 2e-2                                        # unrounded FP32 network
    assert np.abs(out.cpu().numpy()[:, 3]).max() == 0.0


@pytest.mark.parametrize("kind", ["relative", "l2"])
def test_train_step_gradient_and_adam(kind):
    sc = cornell()
    c = RadianceCache(sc, batch=1024, loss=kind)
    lo, inv = c.bounds()
    p = R.init_params(3)
    c.set_params(p)
    n = 1024
    recs = R.random_records(n, lo, lo + 1.0 / inv, seed=4)
    c.train_step(dev(recs).data_ptr(), n)
    torch.cuda.synchronize()
    assert c.counters()[0] == 0
    g = c.gradient()
    loss, wsum = c.loss()
    t, w = recs[:, 16:19].astype(np.float64), recs[:, 19].astype(np.float64)
    lm, gm = R.loss_and_grad(p, R.encode(recs, lo, inv), t, w, kind=kind)
    assert wsum == float(recs[:, 19].sum())
    assert abs(loss - lm) <= 1e-4 * abs(lm)                              # loss
    assert rel_rms(g, gm) <= 1e-2                                        # FP16 model gradient
    _, ge = R.loss_and_grad(p, R.encode(recs, lo, inv, rounded=False), t, w, rounded=False, kind=kind)
    assert rel_rms(g, ge) <= 5e-2                                        # unrounded FP32 gradient
    pa, _, _ = R.adam_step(p, g)
    assert np.abs(c.params() - pa).max() <= 1e-6                         # Adam from the reported gradient


def test_training_reduces_loss_and_save_load():
    sc = cornell()
    c = RadianceCache(sc, batch=4096)
    lo, inv = c.bounds()
    n = 4096
    recs = R.random_records(n, lo, lo + 1.0 / inv, seed=5)
    # a smooth target: radiance = albedo * (0.5 + normalised height)
    recs[:, 16:19] = recs[:, 12:15] * (0.5 + (recs[:, 1:2] - lo[1]) * inv[1])
    d = dev(recs)
    losses = []
    for _ in range(60):
        c.train_step(d.data_ptr(), n)
        losses.append(c.loss()[0])
    assert c.counters()[0] == 0
    assert losses[-1] < 0.2 * losses[0], losses[::10]
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "cache.bin")
        c.save(path)
        c2 = RadianceCache(sc, batch=4096, seed=9)
        c2.load(path)
        assert np.array_equal(c2.params(), c.params())
        # the same next step from the same state
        c.train_step(d.data_ptr(), n)
        c2.train_step(d.data_ptr(), n)
        assert np.array_equal(c2.params(), c.params())


@pytest.mark.parametrize("cache_depth", [1, 2])
def test_zero_cache_equals_truncated_path_tracer(cache_depth):
    sc = cornell()
    c = RadianceCache(sc, cache_depth=cache_depth)
    c.set_params(np.zeros(RadianceCache.param_count(), np.float32))
    w = h = 96
    img = cached(c, sc, w, h, 3, 5)
    ref = plain(sc, w, h, cache_depth, 3)
    assert np.array_equal(img, ref)                                      # bit-identical


@pytest.mark.parametrize("cache_depth", [0, 1, 3])
def test_constant_cache_matches_oracle(cache_depth):
    value = (0.5, 0.25, 0.125)
    sc = cornell()
    c = RadianceCache(sc, cache_depth=cache_depth)
    c.set_params(R.constant_params(value))
    w = h = 64
    frames, depth = 4, 5
    img = cached(c, sc, w, h, frames, depth)
    assert c.counters()[0] == 0 and c.counters()[1] > 0
    ora = CheckerScene(scenes.cornell_box(), "oracle")
    ref = ora.pathtrace_cached(cb.Camera(w, h).flat(), w, h, 0, frames, depth, cache_depth, value).reshape(h, w, 3)
    ok = (np.abs(img - ref) <= np.maximum(1e-4 * np.abs(ref), 1e-6)).all(axis=-1)
    assert ok.mean() >= 0.99, f"{ok.mean():.4f} of pixels within 1e-4"    # per pixel 1e-4
    assert np.abs(img - ref).mean() <= 1e-3 * np.abs(ref).mean()


@pytest.mark.parametrize("specular", [False, True])
def test_constant_cache_specular_matches_oracle(specular):
    """Mirror and glass vertices: continued (default) or answered by the cache."""
    value = (0.5, 0.25, 0.125)
    desc = scenes.material_test_scene(0)
    sc = desc.build()
    c = RadianceCache(sc, cache_depth=1, cache_specular=specular)
    c.set_params(R.constant_params(value))
    w = h = 64
    frames, depth = 4, 5
    img = cached(c, sc, w, h, frames, depth)
    assert c.counters()[0] == 0 and c.counters()[1] > 0
    ora = CheckerScene(desc, "oracle")
    ref = ora.pathtrace_cached(cb.Camera(w, h).flat(), w, h, 0, frames, depth, 1, value,
                               specular=specular).reshape(h, w, 3)
    ok = (np.abs(img - ref) <= np.maximum(1e-4 * np.abs(ref), 1e-6)).all(axis=-1)
    assert ok.mean() >= 0.99, f"{ok.mean():.4f} of pixels within 1e-4"    # per pixel 1e-4
    assert np.abs(img - ref).mean() <= 1e-3 * np.abs(ref).mean()


@pytest.mark.parametrize("cache_depth", [0, 1])
def test_tail_kernel_matches_wavefront(cache_depth):
    """The per-path tail kernel (forced from depth 0) and the wavefront stages
    (tail off) give the same image bit for bit, mirror and glass paths
    included."""
    desc = scenes.material_test_scene(0)
    sc = desc.build()
    w = h = 64
    imgs = []
    for tail in (0, 1 << 30):
        c = RadianceCache(sc, cache_depth=cache_depth)
        c.set_params(R.constant_params((0.5, 0.25, 0.125)))
        c.set_tail_paths(tail)
        imgs.append(cached(c, sc, w, h, 4, 5))
        assert c.counters()[0] == 0
    assert np.array_equal(imgs[0], imgs[1])                              # bit-identical


def test_invalid_arguments_fail_loudly():
    sc = cornell()
    c = RadianceCache(sc, batch=1024)
    d = dev(np.zeros((256, 20), np.float32))
    with pytest.raises(cb.CupbrError):
        c.train_step(d.data_ptr(), 100)                   # not a multiple of 128
    with pytest.raises(cb.CupbrError):
        c.train_step(d.data_ptr(), 2048)                  # above the batch size
    img = torch.zeros((8, 8, 3), device="cuda")
    with pytest.raises(cb.CupbrError):
        c.render(sc, cb.Camera(8, 8), 0, 8, 0, 1, 5, img.data_ptr())       # empty image
    with pytest.raises(cb.CupbrError):
        c.render(sc, cb.Camera(8, 8), 8, 8, 0, 1, 0, img.data_ptr())       # depth 0
    with pytest.raises(cb.CupbrError):
        c.render(sc, cb.Camera(8, 8), 8, 8, 0, 1, 65, img.data_ptr())      # depth above 64
    p = np.zeros(RadianceCache.param_count(), np.float32)
    p[5] = np.nan
    with pytest.raises(cb.CupbrError):
        c.set_params(p)                                   # non-finite weights
    with pytest.raises(ValueError):
        c.set_params(np.zeros(10, np.float32))
    with tempfile.TemporaryDirectory() as tmp:
        bad = os.path.join(tmp, "bad.bin")
        open(bad, "wb").write(b"not a cache")
        with pytest.raises(cb.CupbrError):
            c.load(bad)
    with pytest.raises(cb.CupbrError):
        RadianceCache(sc, batch=100)                      # batch not a multiple of 128
    with pytest.raises(cb.CupbrError):
        RadianceCache(sc, batch=1024, samples_per_frame=1500)
    with pytest.raises(ValueError):
        RadianceCache(sc, loss="huber")
    c.infer(d.data_ptr(), 0, d.data_ptr())                # n = 0: nothing to do
    assert c.counters()[0] == 0


def test_online_training_learns_scene():
    """Online training on the Cornell box: the cache at depth 1 recovers at
    least half of the radiance that paths truncated at depth 1 miss.  The
    per-step relative L2 loss is only checked to stay finite: on single-path
    targets it is heavy-tailed (single steps above 1e3) and its trend is
    noise (the ratio of the last ten steps' median to the first ten's ranged
    over 0.03-2.0 between runs on one B200, the sample order into the
    training batches coming from atomics), while the image criterion held in
    every run."""
    sc = cornell()
    w = h = 128
    c = RadianceCache(sc, cache_depth=1, train_stride=2, batch=8192, samples_per_frame=32768, learning_rate=3e-3,
                      weight_average=0.99)
    c.set_batch_paths(w * h)  # one frame per wavefront: training after every frame
    img = torch.zeros((h, w, 3), device="cuda")
    cam = cb.Camera(w, h)
    losses = []
    for f in range(200):
        c.render(sc, cam, w, h, f, 1, 5, img.data_ptr(), train=True)
        loss, weighted = c.loss()
        if weighted > 0:  # frames that collected too few samples for an Adam step report no loss
            losses.append(loss)
    err, queries, samples = c.counters()
    assert err == 0 and queries > 0 and samples > 0
    assert len(losses) >= 100
    assert np.isfinite(losses).all()
    ref = plain(sc, w, h, 5, 1024).mean(axis=(0, 1))
    trunc = plain(sc, w, h, 1, 256).mean(axis=(0, 1))                    # the light paths ending at depth 1 miss
    got = cached(c, sc, w, h, 64, 5, train=False, frame0=0).mean(axis=(0, 1))
    assert (np.abs(got - ref) < 0.5 * np.abs(trunc - ref)).all(), (got, ref, trunc)   # recovers >= half of it


def test_wait_that_runs_out_is_reported_and_the_cache_stays_usable():
    """Failure detection of the bounded tensor-core waits without a GPU
    fault: the wait probe makes every inference CTA wait 100 us on a barrier
    that nothing arrives on (before any MMA is issued, so no tensor-core work
    is in flight when it gives up).  The call's CTAs count themselves, the
    check reports CUPBR_ERR_TIMEOUT and clears the count, and the next
    inference without the probe gives exactly the result of one made before."""
    sc = cornell()
    c = RadianceCache(sc)
    lo, inv = c.bounds()
    c.set_params(R.init_params(3))
    n = 1000
    recs = dev(R.random_records(n, lo, lo + 1.0 / inv, seed=5, targets=False))
    good = torch.zeros((n, 4), device="cuda")
    c.infer(recs.data_ptr(), n, good.data_ptr())
    c.check()

    out = torch.full((n, 4), -7.0, device="cuda")
    c.set_wait_probe(100_000)
    c.infer(recs.data_ptr(), n, out.data_ptr())
    assert c.counters()[0] > 0
    with pytest.raises(cb.CupbrError) as ei:
        c.check()
    assert ei.value.code == -6  # CUPBR_ERR_TIMEOUT
    assert (out.cpu().numpy() == -7.0).all()  # the CTAs that gave up wrote nothing
    assert c.counters()[0] == 0
    c.check()  # cleared: the cache is usable

    c.set_wait_probe(0)
    again = torch.zeros((n, 4), device="cuda")
    c.infer(recs.data_ptr(), n, again.data_ptr())
    c.check()
    assert torch.equal(again, good)

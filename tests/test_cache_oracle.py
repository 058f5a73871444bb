"""Radiance cache on the CPU: the oracle's cached estimator, the numpy model
of the tensor-core MLP that the GPU tests check against, and the host side of
the C ABI (no GPU).

Bars: the oracle's cached estimator with a zero cache equals its plain path
tracer truncated at the cache depth bit for bit, and is affine in the cache
value (1e-5 relative); the model's gradient matches central differences of
its loss to 1e-5 relative; the constant-cache weights answer their value
exactly.
"""
import numpy as np
import pytest

import cupbr_b200 as cb
from cupbr_b200 import scenes
from cupbr_b200.cache import LAYERS, RadianceCache
from oracle.bridge import CheckerScene

import rc_reference as R

W = H = 24


@pytest.fixture(scope="module")
def ora():
    return CheckerScene(scenes.cornell_box(), "oracle")


def cam():
    return cb.Camera(W, H).flat()


@pytest.mark.parametrize("k", [1, 2, 3])
def test_zero_cache_is_truncated_path_tracer(ora, k):
    img = ora.pathtrace_cached(cam(), W, H, 0, 3, 5, k, (0.0, 0.0, 0.0))
    ref, _ = ora.pathtrace(cam(), W, H, 0, 3, k)
    assert np.array_equal(img, ref)


def test_cached_estimator_is_affine_in_the_cache_value(ora):
    v = np.array([0.5, 0.25, 0.125], np.float32)
    i0 = ora.pathtrace_cached(cam(), W, H, 0, 2, 5, 1, 0 * v).astype(np.float64)
    i1 = ora.pathtrace_cached(cam(), W, H, 0, 2, 5, 1, v).astype(np.float64)
    i2 = ora.pathtrace_cached(cam(), W, H, 0, 2, 5, 1, 2 * v).astype(np.float64)
    d1, d2 = i1 - i0, i2 - i0
    assert (d1 >= 0).all() and d1.sum() > 0
    assert np.abs(d2 - 2 * d1).max() <= 1e-5 * np.abs(d2).max()


def test_cache_depth_zero_answers_primary_hits(ora):
    v = (1.0, 0.5, 0.25)
    img = ora.pathtrace_cached(cam(), W, H, 0, 1, 5, 0, v).reshape(-1, 3)
    # every primary hit in the Cornell box faces the camera and is
    # Lambertian: the image is exactly the cache value
    assert np.array_equal(img, np.tile(np.asarray(v, np.float32), (W * H, 1)))


def test_model_gradient_matches_central_differences():
    rng = np.random.default_rng(0)
    p = R.init_params(7).astype(np.float64)
    recs = R.random_records(16, np.zeros(3), np.ones(3), seed=8)
    X = R.encode(recs, np.zeros(3, np.float32), np.ones(3, np.float32), rounded=False).astype(np.float64)
    t = recs[:, 16:19].astype(np.float64)
    w = recs[:, 19].astype(np.float64)
    y, _ = R.forward(p, X.astype(np.float32), rounded=False)
    den = y.astype(np.float64) ** 2 + 0.01  # the prediction's square is held constant

    def loss(q):
        k, h = 0, X
        for li, (o, i) in enumerate(LAYERS):
            m = q[k:k + o * i].reshape(o, i)
            k += o * i
            z = h @ m.T
            h = np.maximum(z, 0.0) if li + 1 < len(LAYERS) else z
        d = h - t
        return float((w[:, None] * d * d / den).sum() / (3.0 * max(w.sum(), 1.0)))

    _, g = R.loss_and_grad(p, X.astype(np.float32), t, w, rounded=False)
    for idx in rng.choice(len(p), 12, replace=False):
        e = np.zeros_like(p)
        e[idx] = 1e-4
        fd = (loss(p + e) - loss(p - e)) / 2e-4
        assert abs(fd - g[idx]) <= 1e-5 * max(abs(fd), 1e-3) + 1e-7, (idx, fd, g[idx])


def test_constant_params_answer_their_value():
    v = (0.5, 0.25, 0.125)
    recs = R.random_records(50, np.zeros(3), np.ones(3), seed=1, targets=False)
    X = R.encode(recs, np.zeros(3, np.float32), np.ones(3, np.float32))
    y, _ = R.forward(R.constant_params(v), X)
    assert np.array_equal(y, np.tile(np.asarray(v, np.float32), (50, 1)))


def test_host_api_without_gpu():
    assert RadianceCache.param_count() == sum(o * i for o, i in LAYERS) == 22720
    with pytest.raises(cb.CupbrError):
        cb._native.call("cupbr_cache_create", None, None, None)

"""The density-grid medium's oracle (CPU, double precision): the path-replay
adjoint against central differences of the oracle's own forward pass.

The grid medium has no counterpart in the reference, so its oracle is pinned
by calculus instead of golden vectors: with weighted tracking every sample is
a smooth function of the densities and of the albedos / light radiances for
fixed random numbers, so central differences of the forward estimator equal
the adjoint up to rounding (bars below)."""
import dataclasses

import numpy as np
import pytest

import cupbr_b200 as cb
from cupbr_b200 import scenes
from oracle.bridge import CheckerScene

W = H = 16
SPP, DEPTH = 4, 4
BOX = (-1, -1, 1, 1, 1, 3)
MAJ, ALB, G, Q = 3.5, 0.8, 0.3, 0.5


@pytest.fixture(scope="module")
def setup():
    desc = scenes.medium_scene()
    chk = CheckerScene(desc, "oracle")
    grid = scenes.perlin_grid(8, seed=1, sigma_max=3.0).astype(np.float64)
    cam = cb.Camera(W, H).flat()
    wgt = np.random.default_rng(0).random((W * H, 3))
    npar = 1 + 6 * len(desc.objects) + 3 * len(desc.lights)
    gg, gp = chk.medium_backward(grid, BOX, MAJ, ALB, G, Q, cam, W, H, SPP, 0, DEPTH, wgt, npar, precision=64)
    return desc, chk, grid, cam, wgt, gg, gp


def loss(chk, grid, cam, wgt, albedo=ALB):
    img = chk.medium_forward(grid, BOX, MAJ, albedo, G, Q, cam, W, H, SPP, 0, DEPTH, precision=64)
    return float((img * wgt).sum())


def test_forward_is_finite_and_lit(setup):
    _, chk, grid, cam, _, _, _ = setup
    img = chk.medium_forward(grid, BOX, MAJ, ALB, G, Q, cam, W, H, SPP, 0, DEPTH, precision=64)
    assert np.isfinite(img).all() and (img >= 0).all() and img.mean() > 1e-3


def test_density_gradient_matches_central_differences(setup):
    _, chk, grid, cam, wgt, gg, _ = setup
    flat = grid.ravel()
    top = np.argsort(-np.abs(gg).ravel())[:8]
    rng = np.random.default_rng(1)
    rand = rng.choice(np.flatnonzero(flat > 0.05), 8, replace=False)
    h = 1e-4
    scale = np.abs(gg).max()
    assert scale > 0
    for k in np.concatenate([top, rand]):
        gp_, gm_ = flat.copy(), flat.copy()
        gp_[k] += h
        gm_[k] -= h
        fd = (loss(chk, gp_.reshape(grid.shape), cam, wgt) - loss(chk, gm_.reshape(grid.shape), cam, wgt)) / (2 * h)
        # bar: rounding of the differences only (double precision)
        assert abs(gg.ravel()[k] - fd) <= 1e-6 * scale + 1e-5 * abs(fd), (k, gg.ravel()[k], fd)


def _step(v, h):
    """Central-difference endpoints as float32 (the scene and medium
    parameters travel as float32) and their exact distance."""
    a, b = np.float32(v + h), np.float32(v - h)
    return float(a), float(b), float(a) - float(b)


def test_medium_albedo_gradient(setup):
    _, chk, grid, cam, wgt, _, gp = setup
    a, b, step = _step(ALB, 1e-3)
    fd = (loss(chk, grid, cam, wgt, a) - loss(chk, grid, cam, wgt, b)) / step
    assert abs(gp[0] - fd) <= 1e-4 * abs(fd)


@pytest.mark.parametrize("obj,ch", [(0, 0), (2, 0), (3, 1), (5, 2)])
def test_surface_albedo_gradient(setup, obj, ch):
    desc, _, grid, cam, wgt, _, gp = setup
    base = desc.objects[obj].material
    ends = []
    a, b, step = _step(base.albedo_d[ch], 1e-3)
    for v in (a, b):
        d2 = dataclasses.replace(desc, objects=list(desc.objects))
        alb = list(base.albedo_d)
        alb[ch] = v
        d2.objects[obj] = dataclasses.replace(desc.objects[obj], material=dataclasses.replace(base, albedo_d=tuple(alb)))
        ends.append(loss(CheckerScene(d2, "oracle"), grid, cam, wgt))
    fd = (ends[0] - ends[1]) / step
    got = gp[1 + 3 * obj + ch]
    assert abs(got - fd) <= 1e-4 * abs(fd) + 1e-9, (got, fd)


@pytest.mark.parametrize("ch", [0, 1, 2])
def test_light_radiance_gradient(setup, ch):
    desc, _, grid, cam, wgt, _, gp = setup
    base = desc.lights[0]
    ends = []
    a, b, step = _step(base.radiance[ch], 1e-2)
    for v in (a, b):
        rad = list(base.radiance)
        rad[ch] = v
        d2 = dataclasses.replace(desc, lights=[dataclasses.replace(base, radiance=tuple(rad))])
        ends.append(loss(CheckerScene(d2, "oracle"), grid, cam, wgt))
    fd = (ends[0] - ends[1]) / step
    got = gp[1 + 6 * len(desc.objects) + ch]
    assert abs(got - fd) <= 1e-5 * abs(fd), (got, fd)


@pytest.mark.parametrize("obj,ch", [(0, 1), (4, 0), (5, 2)])
def test_emission_gradient(setup, obj, ch):
    """dL/dalbedo_e at surfaces that emit nothing yet: L is linear in the
    emission, so the central difference is exact up to rounding."""
    desc, _, grid, cam, wgt, _, gp = setup
    base = desc.objects[obj].material
    ends = []
    for v in (1e-2, -1e-2):
        d2 = dataclasses.replace(desc, objects=list(desc.objects))
        em = list(base.albedo_e)
        em[ch] = v
        d2.objects[obj] = dataclasses.replace(desc.objects[obj], material=dataclasses.replace(base, albedo_e=tuple(em)))
        ends.append(loss(CheckerScene(d2, "oracle"), grid, cam, wgt))
    fd = (ends[0] - ends[1]) / (float(np.float32(1e-2)) * 2)
    got = gp[1 + 3 * len(desc.objects) + 3 * obj + ch]
    assert abs(got) > 0 and abs(got - fd) <= 1e-5 * abs(fd), (got, fd)


def test_zero_gradient_image_gives_zero_gradients(setup):
    desc, chk, grid, cam, _, _, _ = setup
    npar = 1 + 6 * len(desc.objects) + 3 * len(desc.lights)
    gg, gp = chk.medium_backward(grid, BOX, MAJ, ALB, G, Q, cam, W, H, SPP, 0, DEPTH, np.zeros((W * H, 3)), npar,
                                 precision=64)
    assert not gg.any() and not gp.any()

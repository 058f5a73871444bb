"""GPU parity of the physical estimator (CUPBR_ESTIMATOR_PHYSICAL; no
counterpart in the reference) against the oracle's restatement of it
(oracle.hpp: trace_path_physical, PHYS_MIS; trace_volume_path with the
scene medium's phase value).

Bars: path-traced radiance within 1e-4 relative (abs floor 1e-6) on >= 99 %
of pixels, as for the reference estimator (the rest are paths where a
transcendental function's last bit, here also sincospif in the environment
sample, moved a branch or a texel); VOLUME within 1e-4 on >= 98 %; without
an environment the two estimators are the same estimator, so their images
are bit-identical; the per-path tail kernel leaves the image bit-identical.
"""
import numpy as np
import pytest

import cupbr_b200 as cb
from cupbr_b200 import scenes
from oracle.bridge import CheckerScene

pytestmark = pytest.mark.gpu


def sun_scene():
    desc = scenes.material_test_scene(0, env_size=(96, 48))
    desc.env[10:12, 60:63] = 300.0
    return desc


SCENES = {"mixed": lambda: scenes.material_test_scene(0), "sun": sun_scene}


def within(a, b, rel=1e-4, floor=1e-6):
    return (np.abs(a - b) <= np.maximum(rel * np.abs(b), floor)).all(axis=-1)


def render(sc, w, h, frames, depth, estimator, rr=False, method=cb.RenderingMethod.PATHTRACER, tail=None):
    r = cb.PBRenderer(method)
    r.set_output_size(w, h)
    r.register_scene(sc)
    r.set_method(method)
    r.set_max_trace_depth(depth)
    r.set_russian_roulette(rr)
    r.set_estimator(estimator)
    assert r.get_estimator() == estimator
    if tail is not None:
        r.set_tail_paths(tail)
    cam = cb.Camera(w, h)
    for _ in range(frames):
        r.render(cam)
    img = r.get_output_image().numpy()
    assert r.error_count() == 0
    return img


@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("rr", [False, True])
def test_physical_matches_oracle(name, rr):
    desc = SCENES[name]()
    w, h, frames, depth = 64, 48, 4, 6
    img = render(desc.build(), w, h, frames, depth, "physical", rr)
    ref = CheckerScene(desc, "oracle").pathtrace_physical(cb.Camera(w, h).flat(), w, h, 0, frames, depth, "mis", rr)
    ok = within(img.reshape(-1, 3), ref)
    print(f"physical {name} rr={rr}: {ok.mean():.4f} of pixels within 1e-4 of the oracle")
    assert ok.mean() >= 0.99
    # and it is a different image from the reference estimator's
    assert not np.allclose(img, render(desc.build(), w, h, frames, depth, "reference", rr))


def test_physical_without_environment_is_the_reference_estimator():
    sc = scenes.cornell_box().build()
    a = render(sc, 64, 64, 3, 5, "reference")
    b = render(sc, 64, 64, 3, 5, "physical")
    assert np.array_equal(a, b)                                         # bit-identical


def test_physical_tail_kernel_same_image():
    sc = sun_scene().build()
    a = render(sc, 64, 48, 2, 6, "physical", tail=0)
    b = render(sc, 64, 48, 2, 6, "physical", tail=1 << 30)
    assert np.array_equal(a, b)                                         # bit-identical


def test_physical_1m_triangle_scene_pixels_match_oracle():
    desc = scenes.heightfield_spheres(seed=0)
    sc = desc.build()
    w, h, depth = 1920, 1080, 8
    r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    r.set_output_size(w, h)
    r.register_scene(sc)
    r.set_method(cb.RenderingMethod.PATHTRACER)
    r.set_max_trace_depth(depth)
    r.set_russian_roulette(False)
    r.set_estimator("physical")
    r.render_frames(cb.Camera(w, h), 2)
    img = r.get_output_image().numpy().reshape(-1, 3)
    assert r.error_count() == 0 and np.isfinite(img).all()
    rng = np.random.default_rng(13)
    px = np.sort(rng.choice(w * h, 2000, replace=False)).astype(np.uint32)
    ref = CheckerScene(desc, "oracle").pathtrace_physical(cb.Camera(w, h).flat(), w, h, 0, 2, depth, "mis",
                                                         pixels=px)
    ok = within(img[px], ref)
    print(f"physical 1M-triangle scene: {ok.mean():.4f} of {len(px)} pixels within 1e-4 of the oracle")
    assert ok.mean() >= 0.99


@pytest.mark.parametrize("rr", [False, True])
def test_volume_physical_matches_oracle(rr):
    desc = scenes.volume_test_scene()
    w = h = 48
    img = render(desc.build(), w, h, 3, 6, "physical", rr, method=cb.RenderingMethod.VOLUME)
    ref = CheckerScene(desc, "oracle").volumetrace(cb.Camera(w, h).flat(), w, h, 0, 3, 6, rr, physical=True)
    ok = within(img.reshape(-1, 3), ref)
    print(f"VOLUME physical rr={rr}: {ok.mean():.4f} of pixels within 1e-4 of the oracle")
    assert ok.mean() >= 0.98
    assert not np.allclose(img, render(desc.build(), w, h, 3, 6, "reference", rr, method=cb.RenderingMethod.VOLUME))

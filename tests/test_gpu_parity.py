"""GPU parity: the CUDA path through the C ABI against the reference's own
code run on the host (golden vectors) and against the CPU oracle.

Bars (written next to each assertion):
  * closest-hit object / triangle ids and hit distances: bit-exact
  * visibility: exact
  * path-traced radiance: per pixel within 1e-4 relative (abs floor 1e-6)
    for >= 99% of pixels; the rest are paths where a transcendental function
    (sinf / cosf / powf / acosf / atan2f on the GPU vs the host libm) moved a
    branch decision by one ulp
  * bloom: bit-exact (no transcendental functions)
  * tone map: within 1 LSB everywhere, exact for >= 99.9% of channels
"""
import os

import numpy as np
import pytest

import cupbr_b200 as cb
from cupbr_b200 import scenes
from oracle import bridge
from oracle.bridge import CheckerScene

pytestmark = pytest.mark.gpu

GOLD = os.path.join(os.path.dirname(__file__), "golden")
SCENES = {"cornell": scenes.cornell_box, "mixed": lambda: scenes.material_test_scene(0)}
_built = {}


def scene(name):
    if name not in _built:
        _built[name] = SCENES[name]().build()
    return _built[name]


def golden(name):
    return dict(np.load(os.path.join(GOLD, f"scene_{name}.npz")))


def within(a, b, rel=1e-4, floor=1e-6):
    return (np.abs(a - b) <= np.maximum(rel * np.abs(b), floor)).all(axis=-1)


@pytest.mark.parametrize("name", sorted(SCENES))
def test_closest_hit_bit_exact(name):
    g = golden(name)
    t, obj, tri = scene(name).trace(g["origins"], g["dirs"])
    assert np.array_equal(obj, g["obj"])             # bit-exact object ids
    assert np.array_equal(t, g["t"])                 # bit-exact distances
    o_t, o_obj, o_tri, _, _ = CheckerScene(SCENES[name](), "oracle").trace(g["origins"], g["dirs"])
    assert np.array_equal(tri, o_tri)                # triangle index inside the mesh


@pytest.mark.parametrize("name", sorted(SCENES))
def test_visibility_exact(name):
    g = golden(name)
    vis = scene(name).visible(g["origins"], g["dirs"], g["dist"])
    assert np.array_equal(vis, g["vis"])


def render(sc, w, h, frames, depth, rr=False, method=cb.RenderingMethod.PATHTRACER):
    r = cb.PBRenderer(method)
    r.set_output_size(w, h)
    r.register_scene(sc)
    r.set_method(method)
    r.set_max_trace_depth(depth)
    r.set_russian_roulette(rr)
    cam = cb.Camera(w, h)
    for _ in range(frames):
        r.render(cam)
    img = r.get_output_image().numpy()
    assert r.error_count() == 0
    return r, img


@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("rr", [False, True])
def test_pathtrace_matches_reference(name, rr):
    g = golden(name)
    w, h, depth, frames = int(g["w"]), int(g["h"]), int(g["depth"]), int(g["frames"])
    _, img = render(scene(name), w, h, frames, depth, rr)
    ref = (g["img_rr"] if rr else g["img"]).reshape(h, w, 3)
    ok = within(img, ref)
    assert ok.mean() >= 0.99, f"{ok.mean():.4f} of pixels within 1e-4"
    assert np.abs(img - ref).mean() <= 1e-3 * np.abs(ref).mean()


@pytest.mark.parametrize("name", sorted(SCENES))
def test_resume_from_checkpoint(name):
    g = golden(name)
    w, h, depth, frames = int(g["w"]), int(g["h"]), int(g["depth"]), int(g["frames"])
    r, _ = render(scene(name), w, h, frames, depth)
    # continue two frames from the stored reference image at frame index 4
    host = g["img"].reshape(h, w, 3).astype(np.float32)
    out = r.get_output_image()
    cb._native.call("cupbr_memcpy_h2d", out.ptr, host.ctypes.data, host.nbytes, None)
    r.set_frame_index(frames)
    cam = cb.Camera(w, h)
    r.render(cam)
    r.render(cam)
    img = out.numpy()
    assert within(img, g["img_resume"].reshape(h, w, 3)).mean() >= 0.99


@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("rr", [False, True])
def test_tail_kernel_same_image(name, rr):
    """The per-path tail kernel (forced for every depth) leaves the path
    tracer's image bit-identical."""
    g = golden(name)
    w, h, depth, frames = int(g["w"]), int(g["h"]), int(g["depth"]), int(g["frames"])
    imgs = []
    for tail in (0, 1 << 30):
        r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
        r.set_output_size(w, h)
        r.register_scene(scene(name))
        r.set_method(cb.RenderingMethod.PATHTRACER)
        r.set_max_trace_depth(depth)
        r.set_russian_roulette(rr)
        r.set_tail_paths(tail)
        r.render_frames(cb.Camera(w, h), frames)
        imgs.append(r.get_output_image().numpy())
        assert r.error_count() == 0
    assert np.array_equal(imgs[0], imgs[1])                  # bit-identical


@pytest.mark.parametrize("name", sorted(SCENES))
def test_pipelined_render_same_image(name):
    """Frames traced on the renderer's internal streams (pipelined render())
    with a tone map and readback on the caller's stream between frames give
    the same running mean as synchronous render() calls, bit for bit."""
    import torch
    g = golden(name)
    w, h, depth, frames = int(g["w"]), int(g["h"]), int(g["depth"]), int(g["frames"])
    imgs = []
    for pipelined in (False, True):
        st = torch.cuda.Stream()
        r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
        r.set_output_size(w, h)
        r.register_scene(scene(name))
        r.set_method(cb.RenderingMethod.PATHTRACER)
        r.set_max_trace_depth(depth)
        r.set_russian_roulette(False)
        r.set_stream(st)
        r.set_pipelined(pipelined)
        tm = cb.ToneMapper(cb.ToneMappingType.REINHARD)
        tm.set_stream(st)
        tm.register_image(r.get_output_image())
        cam = cb.Camera(w, h)
        for _ in range(frames + 3):
            r.render(cam)
            tm.tone_map()
            tm.get_render_buffer().numpy(st)
        imgs.append(r.get_output_image().numpy(st))
        assert r.error_count() == 0
    assert np.array_equal(imgs[0], imgs[1])                  # bit-identical


@pytest.mark.parametrize("name", sorted(SCENES))
def test_pipelined_render_frames_same_image(name):
    """render_frames with the wavefronts alternating between the internal
    streams (pipelined) gives the one-stream image bit for bit, with several
    frames per wavefront, a ragged last wavefront and render() calls mixed in."""
    import torch
    g = golden(name)
    w, h, depth = int(g["w"]), int(g["h"]), int(g["depth"])
    imgs = []
    for pipelined in (False, True):
        st = torch.cuda.Stream()
        r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
        r.set_output_size(w, h)
        r.register_scene(scene(name))
        r.set_method(cb.RenderingMethod.PATHTRACER)
        r.set_max_trace_depth(depth)
        r.set_russian_roulette(True)
        r.set_stream(st)
        r.set_batch_paths(3 * w * h)  # 3 frames per wavefront
        r.set_pipelined(pipelined)
        cam = cb.Camera(w, h)
        r.render_frames(cam, 7)
        r.render(cam)
        r.render_frames(cam, 5)
        imgs.append(r.get_output_image().numpy(st))
        assert r.error_count() == 0
    assert np.array_equal(imgs[0], imgs[1])                  # bit-identical


def test_render_deterministic_and_moved_camera_resets():
    sc = scene("cornell")
    _, a = render(sc, 64, 64, 3, 5)
    _, b = render(sc, 64, 64, 3, 5)
    assert np.array_equal(a, b)
    r, _ = render(sc, 64, 64, 3, 5)
    cam = cb.Camera(64, 64)
    cam.set_moved(True)
    r.render(cam)
    assert r.frame_index() == 1


@pytest.mark.parametrize("name", sorted(SCENES))
def test_render_frames_batches_equal_single_frames(name):
    sc = scene(name)
    _, single = render(sc, 40, 24, 5, 6)
    r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    r.set_output_size(40, 24)
    r.register_scene(sc)
    r.set_method(cb.RenderingMethod.PATHTRACER)
    r.set_max_trace_depth(6)
    r.set_batch_paths(40 * 24 * 2)  # two frames per wavefront, then one
    r.render_frames(cb.Camera(40, 24), 5)
    assert r.frame_index() == 5
    assert np.array_equal(r.get_output_image().numpy(), single)


def test_free_function_pathtracing_matches_renderer():
    sc = scene("mixed")
    _, ref = render(sc, 40, 30, 2, 6)
    img = np.zeros((30, 40, 3), np.float32)
    ptr = cb._native.C.c_void_p()
    cb._native.call("cupbr_device_alloc", cb._native.C.byref(ptr), img.nbytes)
    cb._native.call("cupbr_memcpy_h2d", ptr, img.ctypes.data, img.nbytes, None)
    cam = cb.Camera(40, 30)
    for f in range(2):
        cb._native.call("cupbr_pathtracing", sc._h, cb._native.C.byref(cam._c), f, 6, 0, ptr, 40, 30, None)
    cb._native.call("cupbr_memcpy_d2h", img.ctypes.data, ptr, img.nbytes, None)
    cb._native.call("cupbr_stream_synchronize", None)
    cb._native.call("cupbr_device_free", ptr)
    assert np.array_equal(img, ref)


@pytest.mark.parametrize("w,h", [(64, 48), (68, 33), (4, 3), (37, 29), (2, 2)])
def test_bloom_bit_exact(w, h):
    """Widths divisible by 4 take the vectorised kernels, the others the
    per-pixel ones; both are bit-exact."""
    rng = np.random.default_rng(w * h)
    hdr = (rng.random((h, w, 3), dtype=np.float32) * 3.0) ** 2
    hdr[0, 0] = 0
    th = cb.threshold_curve(1.0, 1.0)
    dev = _upload(hdr)
    pp = cb.PostProcessor()
    pp.register_image(dev)
    pp.bloom(th)
    out = pp.get_post_process_buffer().numpy()
    ref = bridge.bloom(hdr, th)
    assert np.array_equal(out, ref)  # bit-exact


@pytest.mark.parametrize("ttype", [cb.ToneMappingType.REINHARD, cb.ToneMappingType.GAMMA])
@pytest.mark.parametrize("h,w", [(33, 65), (34, 68)])
def test_tonemap_and_fused_bloom_tonemap(ttype, h, w):
    rng = np.random.default_rng(5)
    hdr = (rng.random((h, w, 3), dtype=np.float32) * 2.5) ** 3
    hdr[0, :4] = np.array([0.0, 1e-4, 0.0031308, 1e6], np.float32)[:, None]
    dev = _upload(hdr)
    tm = cb.ToneMapper(ttype)
    tm.set_exposure(1.3 if ttype == cb.ToneMappingType.REINHARD else 1.0)
    tm.register_image(dev)
    tm.tone_map()
    out = tm.get_render_buffer().numpy().astype(int)
    ref = bridge.tonemap(hdr, int(ttype), 1.3 if ttype == cb.ToneMappingType.REINHARD else 1.0).astype(int)
    diff = np.abs(out - ref)
    assert diff.max() <= 1 and (diff == 0).mean() >= 0.999   # 1 LSB bar
    th = cb.threshold_curve(0.8, 0.5)
    pp = cb.PostProcessor()
    pp.register_image(dev)
    rgba = _alloc(w, h, 4, np.uint8)
    pp.bloom_tonemap(th, ttype, 1.0, rgba)
    fused = rgba.numpy().astype(int)
    ref2 = bridge.tonemap(bridge.bloom(hdr, th), int(ttype), 1.0).astype(int)
    d2 = np.abs(fused - ref2)
    assert d2.max() <= 1 and (d2 == 0).mean() >= 0.999


@pytest.mark.parametrize("ttype,exposure", [(cb.ToneMappingType.REINHARD, 0.05), (cb.ToneMappingType.REINHARD, 7.5),
                                            (cb.ToneMappingType.REINHARD, 0.0), (cb.ToneMappingType.REINHARD, -1.0),
                                            (cb.ToneMappingType.GAMMA, 1.0)])
def test_tonemap_levels_across_the_float_range(ttype, exposure):
    """The tone map's 8-bit levels over inputs spread across every binade of
    the floats (log-uniform 1e-30 .. 1e30), both signs, zeros, infinities,
    NaN and FLT_MAX, at exposures the level table serves (> 0) and those it
    leaves to the direct formula (0, negative).  Bar: within 1 LSB
    everywhere, exact for >= 99.9 % of channels (as the tone map above)."""
    rng = np.random.default_rng(11)
    h, w = 64, 128
    mag = 10.0 ** rng.uniform(-30, 30, size=(h, w, 3))
    hdr = (mag * np.where(rng.random((h, w, 3)) < 0.1, -1.0, 1.0)).astype(np.float32)
    hdr[:, :8] = rng.random((h, 8, 3), dtype=np.float32) * 4.0      # the range images use
    special = np.array([0.0, -0.0, np.inf, -np.inf, np.nan, np.finfo(np.float32).max, 1e-45, 0.0031308],
                       np.float32)
    hdr[0, 8:16] = special[:, None]
    dev = _upload(hdr)
    tm = cb.ToneMapper(ttype)
    tm.set_exposure(exposure)
    tm.register_image(dev)
    tm.tone_map()
    out = tm.get_render_buffer().numpy().astype(int)
    ref = bridge.tonemap(hdr, int(ttype), exposure).astype(int)
    diff = np.abs(out - ref)
    print(f"exact channels: {(diff == 0).mean():.6f}")
    assert diff.max() <= 1 and (diff == 0).mean() >= 0.999   # 1 LSB bar
    assert np.array_equal(out[0, 8:16], ref[0, 8:16])          # special values exact


def test_tonemap_level_tables_equal_the_formulas_for_every_float():
    """The tone map reads each channel's 8-bit level from tables built on the
    GPU from the formulas (ToneMapper.cu:17-69).  Every 32-bit input, for
    each of the three tables (REINHARD red/green, REINHARD blue, GAMMA):
    the looked-up level equals the formula's, bit for bit, and no bucket was
    left to the formulas."""
    mism = np.zeros(3, np.uint64)
    flagged = np.zeros(3, np.uint32)
    cb._native.call("cupbr_tonemap_verify_levels", mism.ctypes.data, flagged.ctypes.data, None)
    print(f"mismatches {mism.tolist()}, flagged buckets {flagged.tolist()}")
    assert mism.tolist() == [0, 0, 0]
    assert flagged.tolist() == [0, 0, 0]


class _Buf(cb.DeviceImage):
    def __del__(self):
        cb._native.call("cupbr_device_free", self.ptr)


def _alloc(w, h, c, dtype):
    p = cb._native.C.c_void_p()
    cb._native.call("cupbr_device_alloc", cb._native.C.byref(p), w * h * c * np.dtype(dtype).itemsize)
    return _Buf(p.value, w, h, c, dtype)


def _upload(arr):
    h, w, c = arr.shape
    buf = _alloc(w, h, c, arr.dtype)
    a = np.ascontiguousarray(arr)
    cb._native.call("cupbr_memcpy_h2d", buf.ptr, a.ctypes.data, a.nbytes, None)
    cb._native.call("cupbr_stream_synchronize", None)
    return buf


@pytest.fixture(scope="module")
def big_scene():
    desc = scenes.heightfield_spheres(seed=0)
    return desc, desc.build()


def test_1m_triangle_scene_hits_bit_exact(big_scene):
    desc, sc = big_scene
    info = sc.info()
    assert info["triangles"] == 2_024_000 and info["bvh_depth"] < 48
    rng = np.random.default_rng(3)
    n = 3000
    o = np.zeros((n, 3), np.float32)
    o[n // 2:] = rng.uniform([-8, -1, 2], [8, 1, 15], (n - n // 2, 3))
    d = rng.normal(size=(n, 3)).astype(np.float32)
    d[: n // 2, 2] = np.abs(d[: n // 2, 2]) + 0.5
    d[: n // 2, 1] -= 0.4
    t, obj, tri = sc.trace(o, d)
    chk = CheckerScene(desc, "oracle")
    t2, obj2, tri2, _, _ = chk.trace(o, d)
    assert (obj >= 0).mean() > 0.3
    assert np.array_equal(obj, obj2) and np.array_equal(tri, tri2) and np.array_equal(t, t2)


def _first_divergent_bounce(sc, ref_scene, cam, w, h, frames, depth, px):
    """For each pixel of `px`: the smallest trace depth at which this
    library's image and the reference host build's disagree beyond 1e-4
    relative (the same RNG streams truncated at that depth give the radiance
    gathered up to that bounce), or 0 if they agree at every depth."""
    first = np.zeros(len(px), np.int32)
    for k in range(1, depth + 1):
        r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
        r.set_output_size(w, h)
        r.register_scene(sc)
        r.set_method(cb.RenderingMethod.PATHTRACER)
        r.set_max_trace_depth(k)
        r.set_russian_roulette(False)
        r.render_frames(cb.Camera(w, h), frames)
        got = r.get_output_image().numpy().reshape(-1, 3)[px]
        ref, _ = ref_scene.pathtrace(cam, w, h, 0, frames, k, pixels=px)
        bad = ~within(got, ref)
        first[(first == 0) & bad] = k
    return first


@pytest.mark.skipif(bridge.ref_lib() is None, reason="reference host build not present")
def test_1m_triangle_scene_pixels_match_reference_host(big_scene):
    """The 1M-triangle workload at its own resolution and depth (1920x1080,
    depth 8, RR off), 4 frames, on 10,000 seeded pixels against the
    reference's own code compiled for the host (its object BVH over the
    scene's MESH chunks, its geometry, BSDF, light and RNG code).  Bar: >= 99%
    of pixels within 1e-4 relative.  Every divergent pixel is listed with
    the first bounce at which it diverges."""
    desc, sc = big_scene
    w, h, depth, frames = 1920, 1080, 8, 4
    r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    r.set_output_size(w, h)
    r.register_scene(sc)
    r.set_method(cb.RenderingMethod.PATHTRACER)
    r.set_max_trace_depth(depth)
    r.set_russian_roulette(False)
    r.render_frames(cb.Camera(w, h), frames)
    img = r.get_output_image().numpy().reshape(-1, 3)
    assert r.error_count() == 0 and np.isfinite(img).all()
    rng = np.random.default_rng(12)
    px = np.sort(rng.choice(w * h, 10_000, replace=False)).astype(np.uint32)
    ref_scene = CheckerScene(desc, "ref")
    cam = cb.Camera(w, h).flat()
    ref, _ = ref_scene.pathtrace(cam, w, h, 0, frames, depth, pixels=px)
    got = img[px]
    ok = within(got, ref)
    div = px[~ok]
    first = _first_divergent_bounce(sc, ref_scene, cam, w, h, frames, depth, div) if len(div) else []
    print(f"\n1M-triangle scene: {ok.mean():.4f} of {len(px)} pixels within 1e-4 of the reference host build; "
          f"{len(div)} divergent")
    for p, k, g, e in zip(div, first, got[~ok], ref[~ok]):
        print(f"  pixel ({p % w}, {p // w}): first divergent bounce {k}; this library {g}, reference {e}")
    assert ok.mean() >= 0.99, f"{ok.mean():.4f}"


def test_1m_triangle_scene_pixels_match_oracle(big_scene):
    desc, sc = big_scene
    w, h, depth = 1920, 1080, 8
    r, img = render(sc, w, h, 1, depth)
    assert np.isfinite(img).all() and (img >= 0).all()
    rng = np.random.default_rng(11)
    px = np.sort(rng.choice(w * h, 400, replace=False)).astype(np.uint32)
    chk = CheckerScene(desc, "oracle")
    cam = cb.Camera(w, h).flat()
    ref, _ = chk.pathtrace(cam, w, h, 0, 1, depth, pixels=px)
    got = img.reshape(-1, 3)[px]
    ok = within(got, ref)
    assert ok.mean() >= 0.97, f"{ok.mean():.3f}"


def test_1m_triangle_scene_camera_packets_same_image(big_scene):
    """At 1080p the camera rays go through the warp-packet traversal and the
    later bounces through the per-ray one; with every path traced on its
    own by the tail kernel instead, the image is bit-identical."""
    _, sc = big_scene
    w, h = 1920, 1080
    imgs = []
    for tail in (1 << 17, 1 << 30):
        r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
        r.set_output_size(w, h)
        r.register_scene(sc)
        r.set_method(cb.RenderingMethod.PATHTRACER)
        r.set_max_trace_depth(8)
        r.set_russian_roulette(False)
        r.set_tail_paths(tail)
        r.render_frames(cb.Camera(w, h), 2)
        imgs.append(r.get_output_image().numpy())
        assert r.error_count() == 0
    assert np.array_equal(imgs[0], imgs[1])                  # bit-identical


def _pixel_ray(cam, x, y, w, h):
    """Tracing::launchRay without jitter (TracingDetail.h:32-44) in float32."""
    f = np.float32
    rx = f(2.0) * (f(x) / f(w) - f(0.5))
    ry = f(2.0) * (f(y) / f(h) - f(0.5))
    p, ax, ay, az = (np.array(v, np.float32) for v in (cam.position(), cam.x_axis(), cam.y_axis(), cam.z_axis()))
    wp = ((p + az) + rx * ax) + ry * ay
    return p, wp - p


def test_pick_matches_traced_pixel_rays():
    desc = scenes.cornell_box()
    sc = scene("cornell")
    w, h = 48, 40
    cam = cb.Camera(w, h)
    chk = CheckerScene(desc, "oracle")
    xs, ys = np.meshgrid(np.arange(0, w, 5), np.arange(0, h, 4))
    o, d = zip(*(_pixel_ray(cam, x, y, w, h) for x, y in zip(xs.ravel(), ys.ravel())))
    _, obj, _, _, _ = chk.trace(np.array(o), np.array(d))
    hits = 0
    for (x, y), ob in zip(zip(xs.ravel(), ys.ravel()), obj):
        got = sc.pick(cam, int(x), int(y), w, h)
        if ob < 0:
            assert got is None
            continue
        hits += 1
        idx, mat = got
        assert idx == ob
        assert mat.type == desc.objects[ob].material.type
        assert np.allclose(mat.albedo_d.tuple(), desc.objects[ob].material.albedo_d)
    assert hits > 50


def test_update_material_equals_rebuilt_scene():
    desc = scenes.cornell_box()
    sc = desc.build()
    blue = scenes.MaterialDesc(scenes.LAMBERT, albedo_d=(0.1, 0.2, 0.7))
    sc.update_material(2, blue)  # the red wall
    _, img = render(sc, 40, 32, 2, 5)
    desc2 = scenes.cornell_box()
    desc2.objects[2].material = blue
    _, ref = render(desc2.build(), 40, 32, 2, 5)
    assert np.array_equal(img, ref)


@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("rr", [False, True])
def test_persistent_render_frames_same_image(name, rr):
    """render_frames through the persistent kernel (set_persistent) gives the
    wavefront's image bit for bit (with Russian roulette on it falls back to
    the wavefronts, which must then give the same image too)."""
    w, h, frames, depth = 72, 40, 5, 5
    imgs = []
    for persistent in (False, True):
        r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
        r.set_output_size(w, h)
        r.register_scene(scene(name))
        r.set_method(cb.RenderingMethod.PATHTRACER)
        r.set_max_trace_depth(depth)
        r.set_russian_roulette(rr)
        r.set_persistent(persistent)
        r.render_frames(cb.Camera(w, h), frames)
        r.render_frames(cb.Camera(w, h), 2)   # continues the running mean
        imgs.append(r.get_output_image().numpy())
        assert r.error_count() == 0
    assert np.array_equal(imgs[0], imgs[1])                                # bit-identical

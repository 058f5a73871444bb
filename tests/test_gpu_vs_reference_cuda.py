"""The cupbr-b200 kernels against the reference's OWN CUDA path built for
sm_100a with its -use_fast_math flag (oracle/_ref/libref_cuda.so), on the same
B200.  The reference's fast-math arithmetic (approximate division, square
root, sin/cos/exp/pow and free FMA contraction) differs from the IEEE
arithmetic here in the last bits, so the bars are looser than against the
host-compiled reference: radiance within 1e-3 relative for >= 99.9 % of pixels
and 1e-4 for >= 99 % (measured: 99.9 %); bloom within 1e-5 relative; tone map within 2 LSB for
>= 99.9 % of channels.  Skipped where the reference build is absent."""
import numpy as np
import pytest

import cupbr_b200 as cb
from cupbr_b200 import scenes
from oracle import bridge

pytestmark = [pytest.mark.gpu,
              pytest.mark.skipif(not __import__("os").path.exists(bridge.REF_CUDA_LIB),
                                 reason="reference CUDA build not present")]

SCENES = {"cornell": scenes.cornell_box, "mixed": lambda: scenes.material_test_scene(0)}


def within(a, b, rel, floor=1e-6):
    return (np.abs(a - b) <= np.maximum(rel * np.abs(b), floor)).all(axis=-1)


@pytest.mark.parametrize("name", sorted(SCENES))
def test_pathtrace_vs_reference_cuda(name):
    desc = SCENES[name]()
    w = h = 64
    depth = 5 if name == "cornell" else 6
    ref_sc = bridge.RefCudaScene(desc)
    cam = cb.Camera(w, h)
    ref, _ = ref_sc.pathtrace(cam.flat(), w, h, 0, 4, depth)
    sc = desc.build()
    r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    r.set_output_size(w, h)
    r.register_scene(sc)
    r.set_method(cb.RenderingMethod.PATHTRACER)
    r.set_max_trace_depth(depth)
    for _ in range(4):
        r.render(cam)
    img = r.get_output_image().numpy().reshape(-1, 3)
    a3, a4 = within(img, ref, 1e-3).mean(), within(img, ref, 1e-4).mean()
    print(f"{name}: {a4:.4f} of pixels within 1e-4, {a3:.4f} within 1e-3 of the reference CUDA build")
    assert a3 >= 0.999 and a4 >= 0.99


def test_cornell_box_at_its_configuration_vs_reference_cuda():
    """The Cornell-box workload at its stated configuration: 512x512, 64
    frames of 1 spp, max depth 5, Russian roulette off, against the
    reference's own CUDA path on the same GPU.  Bars: >= 99.9% of pixels
    within 1e-3 relative and >= 99% within 1e-4."""
    desc = scenes.cornell_box()
    w = h = 512
    depth, frames = 5, 64
    cam = cb.Camera(w, h)
    ref, _ = bridge.RefCudaScene(desc).pathtrace(cam.flat(), w, h, 0, frames, depth)
    r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    r.set_output_size(w, h)
    r.register_scene(desc.build())
    r.set_method(cb.RenderingMethod.PATHTRACER)
    r.set_max_trace_depth(depth)
    r.set_russian_roulette(False)
    r.render_frames(cam, frames)
    img = r.get_output_image().numpy().reshape(-1, 3)
    assert r.error_count() == 0
    a3, a4 = within(img, ref, 1e-3).mean(), within(img, ref, 1e-4).mean()
    print(f"Cornell 512x512 x 64 frames, depth 5: {a4:.5f} of pixels within 1e-4, {a3:.5f} within 1e-3 "
          f"of the reference CUDA build")
    assert a3 >= 0.999 and a4 >= 0.99


def test_gdpt_reconstruction_alone_bit_exact_vs_reference_cuda():
    """The GDPT reconstruction (init + 50 median passes) given the reference
    CUDA build's own base and one-sided gradient means reproduces that
    build's output and gradient images bit for bit (the passes add, subtract
    and halve only, so fast math changes nothing there)."""
    desc = scenes.material_test_scene(0)
    w, h = 64, 48
    bufs, _ = bridge.RefCudaScene(desc).gradientdomain(cb.Camera(w, h).flat(), w, h, 0, 3, 5)
    dev = {}
    for k in ("base", "gxf", "gxb", "gyf", "gyb"):
        a = np.ascontiguousarray(bufs[k], np.float32)
        p = cb._native.C.c_void_p()
        cb._native.call("cupbr_device_alloc", cb._native.C.byref(p), a.nbytes)
        cb._native.call("cupbr_memcpy_h2d", p.value, a.ctypes.data, a.nbytes, None)
        dev[k] = p.value
    outs = {}
    for k in ("gradient_x", "gradient_y", "temp", "output"):
        p = cb._native.C.c_void_p()
        cb._native.call("cupbr_device_alloc", cb._native.C.byref(p), w * h * 12)
        zero = np.zeros((w * h, 3), np.float32)
        cb._native.call("cupbr_memcpy_h2d", p.value, zero.ctypes.data, zero.nbytes, None)
        outs[k] = p.value
    cb._native.call("cupbr_gdpt_reconstruct", w, h, dev["base"], dev["gxf"], dev["gxb"], dev["gyf"], dev["gyb"],
                    outs["gradient_x"], outs["gradient_y"], outs["temp"], outs["output"], None)
    cb._native.call("cupbr_stream_synchronize", None)
    try:
        for k in ("output", "gradient_x", "gradient_y"):
            got = np.empty((w * h, 3), np.float32)
            cb._native.call("cupbr_memcpy_d2h", got.ctypes.data, outs[k], got.nbytes, None)
            cb._native.call("cupbr_stream_synchronize", None)
            assert np.array_equal(got, bufs[k]), k                       # bit-exact
    finally:
        for p in list(dev.values()) + list(outs.values()):
            cb._native.call("cupbr_device_free", p)


MSCENES = {"volume": scenes.volume_test_scene, "mixed": lambda: scenes.material_test_scene(0)}


def _ours(desc, method, w, h, frames, depth):
    sc = desc.build()
    r = cb.PBRenderer(method)
    r.set_output_size(w, h)
    r.register_scene(sc)
    r.set_method(method)
    r.set_max_trace_depth(depth)
    cam = cb.Camera(w, h)
    for _ in range(frames):
        r.render(cam)
    return r


@pytest.mark.parametrize("name", sorted(MSCENES))
def test_volume_vs_reference_cuda(name):
    desc = MSCENES[name]()
    w = h = 48
    ref, _ = bridge.RefCudaScene(desc).volumetrace(cb.Camera(w, h).flat(), w, h, 0, 3, 6)
    img = _ours(desc, cb.RenderingMethod.VOLUME, w, h, 3, 6).get_output_image().numpy().reshape(-1, 3)
    a3, a4 = within(img, ref, 1e-3).mean(), within(img, ref, 1e-4).mean()
    print(f"VOLUME {name}: {a4:.4f} within 1e-4, {a3:.4f} within 1e-3 of the reference CUDA build")
    assert a3 >= 0.98 and a4 >= 0.95


@pytest.mark.parametrize("name", sorted(MSCENES))
def test_volume_render_frames_equals_renders(name):
    """VOLUME frames batched into multi-frame wavefronts (render_frames, also
    split over several wavefronts by a small path budget) and pipelined
    render() calls give the image of one render() per frame, bit for bit."""
    desc = MSCENES[name]()
    w, h, frames, depth = 40, 32, 7, 6
    sc = desc.build()
    imgs = []
    for budget in (None, 3 * w * h):
        r = cb.PBRenderer(cb.RenderingMethod.VOLUME)
        r.set_output_size(w, h)
        r.register_scene(sc)
        r.set_method(cb.RenderingMethod.VOLUME)
        r.set_max_trace_depth(depth)
        if budget:
            r.set_batch_paths(budget)
        r.render_frames(cb.Camera(w, h), frames)
        imgs.append(r.get_output_image().numpy())
    # pipelined render(): frames traced on the internal streams in turn
    r = cb.PBRenderer(cb.RenderingMethod.VOLUME)
    r.set_output_size(w, h)
    r.register_scene(sc)
    r.set_method(cb.RenderingMethod.VOLUME)
    r.set_max_trace_depth(depth)
    r.set_pipelined(True)
    for _ in range(frames):
        r.render(cb.Camera(w, h))
    imgs.append(r.get_output_image().numpy())
    ref = _ours(desc, cb.RenderingMethod.VOLUME, w, h, frames, depth).get_output_image().numpy()
    for img in imgs:
        assert np.array_equal(img, ref)


@pytest.mark.parametrize("name", sorted(MSCENES))
def test_gdpt_render_frames_equals_renders(name):
    """GRADIENTDOMAIN frames with their paths batched into multi-frame
    wavefronts (render_frames, also split by a small path budget), each frame
    still folded and reconstructed in order, and pipelined render() calls:
    output and gradient images of one render() per frame, bit for bit."""
    desc = MSCENES[name]()
    w, h, frames, depth = 40, 32, 5, 5
    sc = desc.build()
    outs = []
    for budget in (None, 2 * 5 * (w - 2) * (h - 2)):
        r = cb.PBRenderer(cb.RenderingMethod.GRADIENTDOMAIN)
        r.set_output_size(w, h)
        r.register_scene(sc)
        r.set_method(cb.RenderingMethod.GRADIENTDOMAIN)
        r.set_max_trace_depth(depth)
        if budget:
            r.set_batch_paths(budget)
        r.render_frames(cb.Camera(w, h), frames)
        outs.append([r.get_output_image().numpy(), r.get_gradient_x().numpy(), r.get_gradient_y().numpy()])
    # pipelined render(): paths traced on the internal streams in turn
    r = cb.PBRenderer(cb.RenderingMethod.GRADIENTDOMAIN)
    r.set_output_size(w, h)
    r.register_scene(sc)
    r.set_method(cb.RenderingMethod.GRADIENTDOMAIN)
    r.set_max_trace_depth(depth)
    r.set_pipelined(True)
    for _ in range(frames):
        r.render(cb.Camera(w, h))
    outs.append([r.get_output_image().numpy(), r.get_gradient_x().numpy(), r.get_gradient_y().numpy()])
    ref = _ours(desc, cb.RenderingMethod.GRADIENTDOMAIN, w, h, frames, depth)
    want = [ref.get_output_image().numpy(), ref.get_gradient_x().numpy(), ref.get_gradient_y().numpy()]
    for got in outs:
        for a, b in zip(got, want):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("name", sorted(MSCENES))
def test_gdpt_and_raytracer_vs_reference_cuda(name):
    desc = MSCENES[name]()
    w = h = 48
    rs = bridge.RefCudaScene(desc)
    ref, _ = rs.gradientdomain(cb.Camera(w, h).flat(), w, h, 0, 3, 5)
    r = _ours(desc, cb.RenderingMethod.GRADIENTDOMAIN, w, h, 3, 5)
    gx = r.get_gradient_x().numpy().reshape(-1, 3)
    out = r.get_output_image().numpy().reshape(-1, 3)
    ax = within(gx, ref["gradient_x"], 1e-4).mean()
    ao = within(out, ref["output"], 1e-3, 1e-5).mean()
    print(f"GDPT {name}: gradient_x {ax:.4f} within 1e-4, output {ao:.4f} within 1e-3")
    # The reconstruction itself is bit-exact on identical inputs (test
    # above); the output's lower bar is the input differences carried by 50
    # median passes, each of which spreads a pixel's value to its four
    # neighbours.  The input differences: fast-math last bits, and on the
    # all-materials scene the reference's shift paths reading `valid` flags
    # it never initialised (PathData::valid, GradientDomain.cu:13-32, read at
    # :126 past the last vertex of a base path that ended for want of a next
    # direction), which vary from run to run there (observed output
    # fractions 0.844-0.91); here such a vertex is invalid.
    assert ax >= 0.98 and ao >= (0.75 if name == "mixed" else 0.85)
    rt = rs.raytrace(cb.Camera(w, h).flat(), w, h)
    r2 = _ours(desc, cb.RenderingMethod.RAYTRACER, w, h, 1, 5)
    img = r2.get_output_image().numpy().reshape(-1, 3)
    ar = within(img, rt, 1e-4).mean()
    print(f"RAYTRACER {name}: {ar:.4f} within 1e-4")
    assert ar >= 0.99


def test_post_vs_reference_cuda():
    rng = np.random.default_rng(9)
    hdr = (rng.random((96, 128, 3), dtype=np.float32) * 2.0) ** 3
    th = cb.threshold_curve(1.0, 1.0)
    ref = bridge.ref_cuda_bloom(hdr, th)
    ours = bridge.bloom(hdr, th)  # bit-identical to the CUDA kernel (test_gpu_parity)
    assert (np.abs(ours - ref) <= 1e-5 * np.abs(ref) + 1e-7).all()
    for t in (0, 1):
        a = bridge.ref_cuda_tonemap(hdr, t, 1.0).astype(int)
        b = bridge.tonemap(hdr, t, 1.0).astype(int)
        d = np.abs(a - b)
        assert (d <= 2).mean() >= 0.999

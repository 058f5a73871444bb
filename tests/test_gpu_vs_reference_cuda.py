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
    assert ax >= 0.98 and ao >= 0.9
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

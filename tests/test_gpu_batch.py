"""Batched multi-view path tracing (cupbr_batch_*) against per-view
PBRenderer renders.  Bar: bit-exact -- every view of a batch launch equals
`spp` render() calls on its own renderer (same sample streams, same
running-mean arithmetic), across scenes, cameras, sizes, the three modes
(one persistent-kernel launch at every block shape; wavefronts, also split
small; the wavefronts' stages in one cooperative launch, also split small
and at one block per SM) and successive launches; autotuning (BVH leaf sizes included)
leaves the views' images alone and the results unchanged."""
import numpy as np
import pytest

import cupbr_b200 as cb
from cupbr_b200 import scenes

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

DEPTH = 5


def moved(w, h, pos):
    c = cb.Camera(w, h)
    return cb.Camera.from_axes(pos, c.x_axis(), c.y_axis(), c.z_axis())


@pytest.fixture(scope="module")
def setup():
    cornell = scenes.cornell_box().build()
    mixed = scenes.material_test_scene(0).build()
    specs = [(cornell, cb.Camera(48, 40), 48, 40, 3),
             (cornell, moved(32, 32, (0.1, 0.05, -0.2)), 32, 32, 5),
             (mixed, cb.Camera(40, 24), 40, 24, 2),
             (mixed, moved(64, 48, (-0.3, 0.2, 0.1)), 64, 48, 1),
             (cornell, cb.Camera(16, 16), 16, 16, 7)]
    imgs = [torch.zeros((h, w, 3), device="cuda") for (_, _, w, h, _) in specs]
    views = [dict(scene=sc, camera=cam, width=w, height=h, spp=spp, frame0=0, image=img.data_ptr())
             for (sc, cam, w, h, spp), img in zip(specs, imgs)]
    return specs, imgs, views


def reference(spec, frames):
    sc, cam, w, h, _ = spec
    r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    r.set_output_size(w, h)
    r.register_scene(sc)
    r.set_method(cb.RenderingMethod.PATHTRACER)
    r.set_max_trace_depth(DEPTH)
    r.set_russian_roulette(False)
    for _ in range(frames):
        r.render(cam)
    return r.get_output_image().numpy()


def check(specs, imgs, launches):
    torch.cuda.synchronize()
    for spec, img in zip(specs, imgs):
        assert np.array_equal(img.cpu().numpy(), reference(spec, launches * spec[4]))


@pytest.mark.parametrize("mode", ["persistent", "wavefront", "cooperative"])
def test_batch_equals_per_view_renders(setup, mode):
    specs, imgs, views = setup
    for img in imgs:
        img.zero_()
    b = cb.Batch(views, DEPTH)
    assert b.mode()["mode"] == "persistent"  # the default
    b.set_mode(mode)
    info = b.info()
    if mode != "persistent":
        assert info["wavefronts"] == 2 and info["paths"] == sum(w * h * s for (_, _, w, h, s) in specs)
    if mode != "wavefront":
        assert info["kernel_launches"] == 1 and b.mode()["blocks_per_sm"] >= 1
    b.launch()
    check(specs, imgs, 1)
    b.advance()  # the next launch continues every running mean
    b.launch()
    check(specs, imgs, 2)
    assert b.error_count() == 0


@pytest.mark.parametrize("threads", [64, 128, 256])
@pytest.mark.parametrize("blocks", [0, 1])
@pytest.mark.parametrize("packets", [True, False])
def test_persistent_block_shapes(setup, threads, blocks, packets):
    specs, imgs, views = setup
    for img in imgs:
        img.zero_()
    b = cb.Batch(views, DEPTH)
    b.set_mode("persistent", threads, blocks, packets)
    m = b.mode()
    assert m["threads_per_block"] == threads and (blocks == 0 or m["blocks_per_sm"] == 1)
    assert m["camera_packets"] == packets
    b.launch()
    check(specs, imgs, 1)


def test_batch_split_into_small_wavefronts(setup):
    specs, imgs, views = setup
    b = cb.Batch(views, DEPTH)
    b.set_mode("wavefront")
    b.configure(2000, 0.75)  # capacity = one frame of the largest view (3072 paths): views split over wavefronts
    assert b.info()["wavefronts"] >= 5
    for img in imgs:
        img.zero_()
    b.launch()
    check(specs, imgs, 1)


@pytest.mark.parametrize("blocks", [0, 1])
def test_cooperative_small_wavefronts(setup, blocks):
    """Many wavefronts of two scenes in one cooperative launch: every stage
    of every wavefront behind a grid barrier; no barrier times out."""
    specs, imgs, views = setup
    b = cb.Batch(views, DEPTH)
    b.set_mode("cooperative", 256, blocks)
    b.configure(2000)
    assert b.info()["wavefronts"] >= 5 and b.info()["kernel_launches"] == 1
    assert blocks == 0 or b.mode()["blocks_per_sm"] == 1
    for img in imgs:
        img.zero_()
    b.launch()
    check(specs, imgs, 1)
    assert b.error_count() == 0


def test_cooperative_barrier_timeout_is_reported(setup):
    """A grid barrier that one block never reaches (test hook: that block
    leaves before it) ends the launch after the short limit with the timeout
    counted, no fault; the next launch without the hook renders correctly."""
    specs, imgs, views = setup
    b = cb.Batch(views, DEPTH)
    b.set_mode("cooperative")
    b.set_barrier_probe(1_000_000)  # 1 ms
    for img in imgs:
        img.zero_()
    b.launch()
    torch.cuda.synchronize()
    assert b.error_count() >= 1
    b.set_barrier_probe(0)
    for img in imgs:
        img.zero_()
    b.launch()
    check(specs, imgs, 1)
    assert b.error_count() == 0


def test_cooperative_shape_is_checked(setup):
    _, _, views = setup
    b = cb.Batch(views, DEPTH)
    with pytest.raises(cb.CupbrError):
        b.set_mode("cooperative", 128)


def test_autotune_leaves_images_alone(setup):
    specs, imgs, views = setup
    b = cb.Batch(views, DEPTH)
    b.launch()
    torch.cuda.synchronize()
    before = [img.clone() for img in imgs]
    ms = b.autotune()
    torch.cuda.synchronize()
    assert ms > 0
    for a, c in zip(before, imgs):
        assert torch.equal(a, c)
    m = b.mode()
    if m["mode"] != "persistent":
        assert b.info()["batch_paths"] in (1 << 21, 1 << 22, 1 << 23, 1 << 24, 1 << 25)
    else:
        assert m["threads_per_block"] in (64, 128, 256)


def test_autotune_with_bvh_leaf_sizes_keeps_results(setup):
    """Rebuilding the scenes' BVHs at other leaf sizes changes no hit, so
    the tuned batch still gives every view its render() image."""
    specs, imgs, views = setup
    b = cb.Batch(views, DEPTH)
    assert b.autotune(bvh_leaf=True) > 0
    for img in imgs:
        img.zero_()
    b.launch()
    check(specs, imgs, 1)


def test_other_batch_follows_a_scene_recommit(setup):
    """A batch whose scenes another batch's autotuner re-committed (new BVH,
    new device buffers) rebuilds its tables at its next launch and still
    gives every view its render() image."""
    specs, imgs, views = setup
    first = cb.Batch(views, DEPTH)
    second = cb.Batch(views, DEPTH)
    assert second.autotune(bvh_leaf=True) > 0  # may re-commit the scenes
    for img in imgs:
        img.zero_()
    first.launch()
    check(specs, imgs, 1)

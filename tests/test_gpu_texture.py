"""Albedo textures and their adjoint (no counterpart in the reference).

Bars: textured renders within 1e-4 relative per pixel of the oracle's
textured estimator on >= 99 % of pixels (as the untextured path tracer);
a batch of textured views bit-identical to per-view render() calls; the
texture adjoint (cupbr_batch_backward, path replay) within 1e-3 relative of
central differences of an L2 image loss on the texels with the largest
gradients and on random texels (with common random numbers every path is
the same for every texture, and the image is linear in a texel unless a
path meets the texel twice, whose quadratic term central differences
cancel, so the differences are exact up to float rounding).
"""
import numpy as np
import pytest

import cupbr_b200 as cb
from cupbr_b200 import scenes
from oracle.bridge import CheckerScene

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def within(a, b, rel=1e-4, floor=1e-6):
    return (np.abs(a - b) <= np.maximum(rel * np.abs(b), floor)).all(axis=-1)


def textured_mixed():
    d = scenes.material_test_scene(0)
    d.texture = scenes.albedo_texture(128, seed=7)
    d.objects[0].tex_frame = ((-2.0, -1.0, 1.0), (4.0, 0.0, 0.0), (0.0, 0.0, 4.0))   # the ground plane
    d.objects[1].tex_frame = ((-1.6, -0.9, 4.5), (3.2, 0.0, 0.0), (0.0, 2.2, 0.0))   # the back quad
    return d


SCENES = {"cornell": lambda: scenes.with_texture(scenes.cornell_variant(2), 256, seed=5), "mixed": textured_mixed}


@pytest.mark.parametrize("name", sorted(SCENES))
@pytest.mark.parametrize("estimator", ["reference", "physical"])
def test_textured_render_matches_oracle(name, estimator):
    desc = SCENES[name]()
    w, h, frames, depth = 64, 48, 4, 5
    r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    r.set_output_size(w, h)
    r.register_scene(desc.build())
    r.set_method(cb.RenderingMethod.PATHTRACER)
    r.set_max_trace_depth(depth)
    r.set_russian_roulette(False)
    r.set_estimator(estimator)
    r.render_frames(cb.Camera(w, h), frames)
    img = r.get_output_image().numpy().reshape(-1, 3)
    chk = CheckerScene(desc, "oracle")
    cam = cb.Camera(w, h).flat()
    if estimator == "reference":
        ref, _ = chk.pathtrace(cam, w, h, 0, frames, depth)
    else:
        ref = chk.pathtrace_physical(cam, w, h, 0, frames, depth, "mis")
    ok = within(img, ref)
    print(f"textured {name} ({estimator}): {ok.mean():.4f} of pixels within 1e-4 of the oracle")
    assert ok.mean() >= 0.99
    # the texture is used: the untextured scene renders differently
    plain = SCENES[name]()
    plain.texture = None
    ref2, _ = CheckerScene(plain, "oracle").pathtrace(cam, w, h, 0, frames, depth)
    assert not np.allclose(ref, ref2)


def render_views(specs, depth):
    out = []
    for sc, cam, w, h, spp in specs:
        r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
        r.set_output_size(w, h)
        r.register_scene(sc)
        r.set_method(cb.RenderingMethod.PATHTRACER)
        r.set_max_trace_depth(depth)
        r.set_russian_roulette(False)
        for _ in range(spp):
            r.render(cam)
        out.append(r.get_output_image().numpy())
    return out


def test_textured_batch_equals_renders():
    a = scenes.with_texture(scenes.cornell_variant(1), 256, seed=11).build()
    b = textured_mixed().build()
    specs = [(a, cb.Camera(40, 32), 40, 32, 3), (b, cb.Camera(48, 24), 48, 24, 2), (a, cb.Camera(24, 24), 24, 24, 4)]
    imgs = [torch.zeros((h, w, 3), device="cuda") for (_, _, w, h, _) in specs]
    batch = cb.Batch([dict(scene=sc, camera=cam, width=w, height=h, spp=spp, frame0=0, image=img.data_ptr())
                      for (sc, cam, w, h, spp), img in zip(specs, imgs)], 5)
    batch.launch()
    torch.cuda.synchronize()
    for img, ref in zip(imgs, render_views(specs, 5)):
        assert np.array_equal(img.cpu().numpy(), ref)                     # bit-identical


class FD:
    """A small textured batch with an L2 loss against a target rendered from
    a perturbed texture."""

    def __init__(self):
        self.desc = scenes.with_texture(scenes.cornell_variant(3), 16, seed=13)
        self.scene = self.desc.build()
        self.tex = torch.as_tensor(self.scene.albedo_texture(), device="cuda")  # (16, 16, 4) view
        self.depth = 4
        base = cb.Camera(32, 40)
        moved = cb.Camera.from_axes((0.2, 0.1, 0.0), base.x_axis(), base.y_axis(), base.z_axis())
        self.specs = [(cb.Camera(48, 48), 48, 48, 8), (moved, 32, 40, 8)]
        self.imgs = [torch.zeros((h, w, 3), device="cuda") for (_, w, h, _) in self.specs]
        self.batch = cb.Batch([dict(scene=self.scene, camera=cam, width=w, height=h, spp=spp, frame0=0,
                                    image=img.data_ptr()) for (cam, w, h, spp), img in zip(self.specs, self.imgs)],
                              self.depth)
        # target: the same views with the texture scaled by (1 +- 10 %)
        base = self.tex.clone()
        g = torch.Generator(device="cuda").manual_seed(3)
        self.tex[..., :3] *= 1.0 + 0.1 * (2.0 * torch.rand(self.tex[..., :3].shape, generator=g, device="cuda") - 1.0)
        self.targets = [t.clone() for t in self.render()]
        self.tex.copy_(base)

    def render(self):
        for img in self.imgs:
            img.zero_()
        self.batch.launch()
        torch.cuda.synchronize()
        return self.imgs

    def loss(self):
        return sum(0.5 * float(((img.double() - t.double()) ** 2).sum()) for img, t in zip(self.render(), self.targets))


def test_texture_adjoint_matches_central_differences():
    fd = FD()
    imgs = fd.render()
    grads = [(img - t).contiguous() for img, t in zip(imgs, fd.targets)]
    fd.batch.backward([g.data_ptr() for g in grads])
    torch.cuda.synchronize()
    adj = fd.batch.texture_gradient(fd.scene).numpy()                    # (16, 16, 3)
    assert np.isfinite(adj).all() and np.abs(adj).max() > 0
    flat = np.abs(adj).reshape(-1)
    order = np.argsort(-flat)
    rng = np.random.default_rng(5)
    picks = list(order[:8]) + list(rng.choice(order[:len(order) // 2], 4, replace=False))
    h = 0.02
    worst = 0.0
    for k in picks:
        y, x, c = np.unravel_index(k, adj.shape)
        v0 = float(fd.tex[y, x, c])
        fd.tex[y, x, c] = v0 + h
        lp = fd.loss()
        fd.tex[y, x, c] = v0 - h
        lm = fd.loss()
        fd.tex[y, x, c] = v0
        num = (lp - lm) / (2.0 * h)
        rel = abs(adj[y, x, c] - num) / max(abs(num), 1e-12)
        worst = max(worst, rel)
        print(f"texel ({x}, {y}) channel {c}: adjoint {adj[y, x, c]:.6e}, central difference {num:.6e}, rel {rel:.2e}")
        assert rel <= 1e-3                                                   # 1e-3 relative
    print(f"worst relative difference {worst:.2e}")


def test_texture_adjoint_accumulates():
    fd = FD()
    imgs = fd.render()
    grads = [(img - t).contiguous() for img, t in zip(imgs, fd.targets)]
    fd.batch.backward([g.data_ptr() for g in grads])
    one = fd.batch.texture_gradient(fd.scene).numpy().copy()
    fd.batch.backward([g.data_ptr() for g in grads], accumulate=True)
    two = fd.batch.texture_gradient(fd.scene).numpy()
    assert np.allclose(two, 2.0 * one, rtol=1e-5, atol=1e-9)
    fd.batch.backward([g.data_ptr() for g in grads])  # accumulate off: set, not added
    assert np.allclose(fd.batch.texture_gradient(fd.scene).numpy(), one, rtol=1e-5, atol=1e-9)

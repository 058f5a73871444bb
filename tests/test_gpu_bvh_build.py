"""The device BVH builder (bvh_gpu.cu) against the host builder
(bvh_build.cpp).

Bar: bit-exact -- the 4-wide node array the traversal kernels read and the
primitive slot order (per primitive key) are identical; node / leaf counts
and depth equal; the SAH statistic (a double sum taken in another order)
within 1e-9 relative.  Cases cover every path of the device build: large
nodes binned across the GPU (the 2M-triangle heightfield), one-CTA
subtrees, the object-median fallback of a large node (done on the host)
and of a small one (in the CTA), several primitive types joined under one
root, a single-primitive scene (the wrapped leaf root) and an empty one.
"""
import numpy as np
import pytest

import cupbr_b200 as cb
from cupbr_b200 import scenes
from cupbr_b200.scenes import MESH, PLANE, QUAD, SPHERE, TRIANGLE, MaterialDesc, ObjectDesc, SceneDesc

pytestmark = pytest.mark.gpu


def _same_bvh(desc, **params):
    a = desc.build(bvh_params={"builder": "host", **params})
    b = desc.build(bvh_params={"builder": "device", **params})
    ia, ib = a.info(), b.info()
    for k in ("bvh_nodes", "bvh_leaves", "bvh_depth", "triangles", "spheres", "quads", "planes"):
        assert ia[k] == ib[k], k
    assert ib["bvh_sah_cost"] == pytest.approx(ia["bvh_sah_cost"], rel=1e-9)
    na, nb = a.bvh_nodes(), b.bvh_nodes()
    assert na.shape == nb.shape
    assert np.array_equal(na.view(np.uint32), nb.view(np.uint32))       # bit-exact nodes
    assert np.array_equal(a.key_slots(), b.key_slots())                  # same leaf order
    return a, b


def _identical_triangles(n, at=(0.0, 0.0, 3.0)):
    """n copies of one triangle: every centroid equal, so no SAH split."""
    v = np.array([[0, 0, 0], [0.5, 0, 0], [0, 0.5, 0]], np.float32)
    verts = np.tile(v, (n, 1))
    idx = np.arange(3 * n, dtype=np.uint32).reshape(n, 3)
    return ObjectDesc(MESH, MaterialDesc(), vertices=verts, indices=idx, position=at)


def test_cornell_and_mixed_scenes():
    for desc in (scenes.cornell_box(), scenes.material_test_scene(0)):
        _same_bvh(desc)


def test_bvh_parameters():
    desc = scenes.material_test_scene(0)
    for params in ({"max_leaf_size": 1}, {"max_leaf_size": 8, "traversal_cost": 0.5}, {"top_bfs_levels": 0},
                   {"top_bfs_levels": 8}):
        _same_bvh(desc, **params)


def test_heightfield_2m_triangles():
    desc = scenes.heightfield_spheres(seed=1)
    a, b = _same_bvh(desc)
    assert b.info()["triangles"] == 2_024_000


def test_identical_centroids_large_and_small():
    for n in (300, 5000):  # one-CTA median / large-node median on the host
        desc = SceneDesc()
        desc.add(_identical_triangles(n))
        desc.add(ObjectDesc(SPHERE, MaterialDesc(), p0=(0.0, 0.0, 4.0), radius=0.5))
        _same_bvh(desc)


def test_single_primitive_and_empty_scene():
    d = SceneDesc()
    d.add(ObjectDesc(SPHERE, MaterialDesc(), p0=(0.0, 0.0, 3.0), radius=1.0))
    _same_bvh(d)
    t = SceneDesc()
    t.add(ObjectDesc(TRIANGLE, MaterialDesc(), vertices=np.array([[0, 0, 2], [1, 0, 2], [0, 1, 2]], np.float32)))
    _same_bvh(t)
    p = SceneDesc()
    p.add(ObjectDesc(PLANE, MaterialDesc(), p0=(0.0, -1.0, 0.0), p1=(0.0, 1.0, 0.0)))
    _same_bvh(p)


def test_random_soup():
    rng = np.random.default_rng(5)
    desc = SceneDesc()
    for k in range(6):
        n = int(rng.integers(1, 3000))
        c = rng.uniform(-3, 3, size=(n, 1, 3)).astype(np.float32)
        tri = (c + rng.normal(scale=0.05 * (k + 1), size=(n, 3, 3))).astype(np.float32)
        desc.add(ObjectDesc(MESH, MaterialDesc(), vertices=tri.reshape(-1, 3),
                            indices=np.arange(3 * n, dtype=np.uint32).reshape(n, 3), position=(0.0, 0.0, 6.0)))
    for k in range(40):
        desc.add(ObjectDesc(SPHERE, MaterialDesc(), p0=tuple(rng.uniform(-2, 2, 3) + [0, 0, 6]),
                            radius=float(rng.uniform(0.05, 0.4))))
    desc.add(ObjectDesc(QUAD, MaterialDesc(), p0=(0.0, -2.0, 6.0), p1=(0.0, 1.0, 0.0), p2=(2.0, 0.0, 0.0),
                        p3=(0.0, 0.0, 2.0)))
    a, b = _same_bvh(desc)
    # and the two scenes render the same image
    imgs = []
    for s in (a, b):
        r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
        r.set_output_size(96, 64)
        r.register_scene(s)
        r.set_method(cb.RenderingMethod.PATHTRACER)
        r.set_max_trace_depth(4)
        r.render_frames(cb.Camera(96, 64), 2)
        imgs.append(r.get_output_image().numpy())
        assert r.error_count() == 0
    assert np.array_equal(imgs[0], imgs[1])


def test_invalid_builder_name():
    with pytest.raises(ValueError):
        scenes.cornell_box().build(bvh_params={"builder": "gpu"})

"""Generate the golden vectors that pin the CPU oracle.

Every value here comes from the REFERENCE's own code compiled for the host
(oracle/_ref/libref_host.so, built by oracle/build_oracle.py from the
reference sources): Math::tea / rnd, Material::sampleDirection / brdf,
Light::sample, Tracing::traceRay / traceVisibility through its object BVH,
and the path-tracing kernel body run per pixel.  The scenes are the seeded
generators of cupbr_b200.scenes, so the GPU tests can rebuild them without
the reference tree.

Run in a checkout where the reference tree is present:
    python oracle/build_oracle.py && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from cupbr_b200 import scenes  # noqa: E402
from oracle.bridge import CheckerScene, ref_lib, _ptr  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def rays_for(desc: scenes.SceneDesc, n: int, seed: int, lo, hi):
    rng = np.random.default_rng(seed)
    o = rng.uniform(lo, hi, (n, 3)).astype(np.float32)
    d = rng.normal(size=(n, 3)).astype(np.float32)
    # a few axis-aligned and near-axis directions (slab-test edge cases)
    d[: n // 16] = 0
    d[np.arange(n // 16), rng.integers(0, 3, n // 16)] = rng.choice([-1.0, 1.0], n // 16)
    d[n // 16: n // 8] += (rng.normal(size=(n // 8 - n // 16, 3)) * 1e-6).astype(np.float32)
    return o, d


def material_cases(rng):
    M = scenes.MaterialDesc
    return [M(scenes.LAMBERT, albedo_d=(0.7, 0.5, 0.3)),
            M(scenes.PHONG, albedo_d=(0.2, 0.3, 0.8), albedo_s=(1, 1, 1), shininess=51.2),
            M(scenes.MIRROR, albedo_s=(0.9, 0.8, 0.7)),
            M(scenes.GLASS, albedo_s=(1, 1, 1), eta=1.5),
            M(scenes.GGX, albedo_s=(1.0, 0.8, 0.9), roughness=0.1),
            M(scenes.GGX, albedo_s=(0.5, 0.6, 0.7), roughness=0.6),
            M(scenes.VOLUME, interface_glass=1, eta=1.33),
            M(scenes.VOLUME, interface_glass=0)]


def unit(v):
    return (v / np.linalg.norm(v, axis=-1, keepdims=True)).astype(np.float32)


def main() -> int:
    ref = ref_lib()
    if ref is None:
        print("reference host build missing: run python oracle/build_oracle.py first", file=sys.stderr)
        return 1
    rng = np.random.default_rng(1234)

    # ---- RNG known answers (FunctionsDetail.h:70-98)
    pairs = rng.integers(0, 2**32, size=(256, 2), dtype=np.uint64).astype(np.uint32)
    pairs[:8] = [[0, 0], [1, 0], [0, 1], [511, 63], [262143, 0], [2**32 - 1, 2**32 - 1], [12345, 7], [7, 12345]]
    tea = np.array([ref.ref_tea4(int(a), int(b)) for a, b in pairs], dtype=np.uint32)
    seeds = np.array([0, 1, 0xDEADBEEF, 2**32 - 1], dtype=np.uint32)
    draws = np.zeros((len(seeds), 64), np.float32)
    states = np.zeros((len(seeds), 64), np.uint32)
    for i, s in enumerate(seeds):
        ref.ref_rnd_stream(int(s), 64, _ptr(draws[i]), _ptr(states[i]))
    np.savez_compressed(os.path.join(OUT, "rng.npz"), pairs=pairs, tea=tea, seeds=seeds, draws=draws, states=states)

    # ---- BSDF sampling / evaluation known answers (MaterialDetail.h:35-313)
    mats = material_cases(rng)
    n = 128
    mat_flat = np.stack([m.flat() for m in mats])
    inc = unit(rng.normal(size=(len(mats), n, 3)))
    nrm = unit(rng.normal(size=(len(mats), n, 3)))
    out = unit(rng.normal(size=(len(mats), n, 3)))
    sd = rng.integers(0, 2**32, size=(len(mats), n), dtype=np.uint64).astype(np.uint32)
    samp = np.zeros((len(mats), n, 4), np.float32)
    sout = np.zeros((len(mats), n), np.uint32)
    brdf = np.zeros((len(mats), n, 3), np.float32)
    for i in range(len(mats)):
        m = np.ascontiguousarray(mat_flat[i])
        for k in range(n):
            so = np.zeros(1, np.uint32)
            ref.ref_sample_direction(_ptr(m), int(sd[i, k]), _ptr(inc[i, k]), _ptr(nrm[i, k]), _ptr(samp[i, k]), _ptr(so))
            sout[i, k] = so[0]
            # evaluate at the sampled direction for half the cases (delta lobes), random otherwise
            o = samp[i, k, :3].copy() if k % 2 == 0 else out[i, k]
            ref.ref_brdf(_ptr(m), _ptr(inc[i, k]), _ptr(np.ascontiguousarray(o)), _ptr(nrm[i, k]), _ptr(brdf[i, k]))
            if k % 2 == 0:
                out[i, k] = o
    np.savez_compressed(os.path.join(OUT, "bsdf.npz"), mats=mat_flat, inc=inc, nrm=nrm, out=out, seeds=sd,
                        sample=samp, seed_out=sout, brdf=brdf)

    # ---- light sampling (LightDetail.h:8-52)
    lights = [scenes.LightDesc(scenes.POINT, position=(0.5, 1.5, 1.5), intensity=(2, 2, 1.8)),
              scenes.LightDesc(scenes.AREA, position=(0, 0.99, 2), radiance=(17, 12, 4), half_extend1=(0.125, 0, 0),
                               half_extend2=(0, 0, 0.125)),
              scenes.LightDesc(scenes.AREA, position=(-0.5, 1.6, 2.5), radiance=(6, 5, 4), half_extend1=(0.3, 0, 0),
                               half_extend2=(0, 0.05, 0.2))]
    lf = np.stack([l.flat() for l in lights])
    P = rng.uniform(-1, 1, (len(lights), n, 3)).astype(np.float32)
    P[..., 2] += 2
    ls = rng.integers(0, 2**32, size=(len(lights), n), dtype=np.uint64).astype(np.uint32)
    lrad = np.zeros((len(lights), n, 3), np.float32)
    ldir = np.zeros((len(lights), n, 3), np.float32)
    ldist = np.zeros((len(lights), n), np.float32)
    lso = np.zeros((len(lights), n), np.uint32)
    for i in range(len(lights)):
        l = np.ascontiguousarray(lf[i])
        for k in range(n):
            so = np.zeros(1, np.uint32)
            dd = np.zeros(1, np.float32)
            ref.ref_light_sample(_ptr(l), int(ls[i, k]), _ptr(P[i, k]), _ptr(lrad[i, k]), _ptr(ldir[i, k]), _ptr(dd),
                                 _ptr(so))
            ldist[i, k], lso[i, k] = dd[0], so[0]
    np.savez_compressed(os.path.join(OUT, "light.npz"), lights=lf, P=P, seeds=ls, radiance=lrad, dir=ldir,
                        dist=ldist, seed_out=lso)

    # ---- closest hit / visibility / path tracing on the seeded scenes
    cases = {"cornell": (scenes.cornell_box(), (-0.98, -0.98, 1.02), (0.98, 0.98, 2.98), 5),
             "mixed": (scenes.material_test_scene(0), (-2.0, -0.9, 1.0), (2.0, 1.8, 4.4), 6)}
    for name, (desc, lo, hi, depth) in cases.items():
        sc = CheckerScene(desc, "ref")
        o, d = rays_for(desc, 4096, 7, lo, hi)
        t, obj, _, Ph, Nh = sc.trace(o, d)
        dist = (rng.uniform(0.0, 3.0, len(o))).astype(np.float32)
        dist[::7] = np.inf
        vis = sc.visible(o, d, dist)
        cam = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1], np.float32)
        w = h = 48
        img, counts = sc.pathtrace(cam, w, h, 0, 4, depth, rr=False)
        img_rr, _ = sc.pathtrace(cam, w, h, 0, 4, depth, rr=True)
        # resume from frame 4 on top of the 4-frame image: frames 4..5
        img_resume, _ = sc.pathtrace(cam, w, h, 4, 2, depth, rr=False, img=img.copy())
        np.savez_compressed(os.path.join(OUT, f"scene_{name}.npz"), origins=o, dirs=d, t=t, obj=obj, P=Ph, N=Nh,
                            dist=dist, vis=vis, cam=cam, w=w, h=h, depth=depth, frames=4, img=img, img_rr=img_rr,
                            img_resume=img_resume, rays=np.array(counts, np.uint64))
        print(name, "hits", int((obj >= 0).sum()), "visible", int(vis.sum()), "mean radiance", float(img.mean()))

    # ---- VOLUME method (VolumeRenderer.cu:214-310) and GRADIENTDOMAIN frames
    # (GradientDomain.cu:160-246), kernel bodies restated over the reference's
    # own Tracing / Material / Light / BVH code
    cam = np.array([0, 0, 0, 1, 0, 0, 0, 1, 0, 0, 0, 1], np.float32)
    w = h = 40
    vcases = {"volume": scenes.volume_test_scene(), "mixed": scenes.material_test_scene(0),
              "cornell": scenes.cornell_box()}
    for name, desc in vcases.items():
        sc = CheckerScene(desc, "ref")
        vol = sc.volumetrace(cam, w, h, 0, 3, 6)
        vol_rr = sc.volumetrace(cam, w, h, 0, 3, 6, rr=True)
        gd = sc.gdpt(cam, w, h, 0, 3, 5)
        rt = sc.raytrace(cam, w, h)
        np.savez_compressed(os.path.join(OUT, f"methods_{name}.npz"), cam=cam, w=w, h=h, frames=3, vol_depth=6,
                            gd_depth=5, volume=vol, volume_rr=vol_rr, gd_base=gd[0], gd_gxf=gd[1], gd_gxb=gd[2],
                            gd_gyf=gd[3], gd_gyb=gd[4], raytrace=rt)
        print(name, "volume mean", float(vol.mean()), "gdpt base mean", float(gd[0].mean()))
    return 0


if __name__ == "__main__":
    sys.exit(main())

"""ctypes bridge to the CPU checkers -- TEST INFRASTRUCTURE ONLY.

Loads oracle/liboracle.so (the C++ restatement) and, when it was built,
oracle/_ref/libref_host.so (the reference's own code compiled for the host).
Only tests/, __graft_entry__.smoke() and bench.py's CPU legs import this.
Scenes are given as cupbr_b200.scenes.SceneDesc objects (plain data).
"""
from __future__ import annotations

import ctypes as C
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_LIB = os.path.join(HERE, "liboracle.so")
REF_HOST_LIB = os.path.join(HERE, "_ref", "libref_host.so")

_P = C.c_void_p


def _ptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data


def _load_oracle() -> C.CDLL:
    if not os.path.exists(ORACLE_LIB):
        from . import build_oracle  # noqa: F401  (build on demand where a compiler exists)
        build_oracle.build_oracle()
    lib = C.CDLL(ORACLE_LIB)
    sig = {
        "ora_scene_new": ([C.c_int], _P), "ora_scene_free": ([_P], None),
        "ora_scene_add_object": ([_P, C.c_int, _P, C.c_float, _P, _P, C.c_int, _P], None),
        "ora_scene_add_light": ([_P, _P], None), "ora_scene_set_env": ([_P, _P, C.c_uint32, C.c_uint32], None),
        "ora_scene_set_volume": ([_P, _P, _P, C.c_float], None), "ora_scene_finalize": ([_P], None),
        "ora_scene_dfs_order": ([_P, _P, C.c_int], C.c_int),
        "ora_trace": ([_P, C.c_int, _P, _P, _P, _P, _P, _P, _P, C.c_int], None),
        "ora_visible": ([_P, C.c_int, _P, _P, _P, _P, C.c_int], None),
        "ora_pathtrace_f32": ([_P, _P, C.c_uint32, C.c_uint32, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                               C.c_int, _P, C.c_int, _P], None),
        "ora_pathtrace_f64": ([_P, _P, C.c_uint32, C.c_uint32, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                               C.c_int, _P, C.c_int, _P], None),
        "ora_pathtrace_cached_f32": ([_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                      _P, C.c_int, _P, C.c_int], None),
        "ora_tea4": ([C.c_uint32, C.c_uint32], C.c_uint32), "ora_rnd_stream": ([C.c_uint32, C.c_int, _P, _P], None),
        "ora_sample_direction": ([_P, C.c_uint32, _P, _P, _P, _P], None), "ora_brdf": ([_P, _P, _P, _P, _P], None),
        "ora_light_sample": ([_P, C.c_uint32, _P, _P, _P, _P, _P], None),
        "ora_tonemap": ([_P, C.c_uint64, C.c_int, C.c_float, _P], None),
        "ora_bloom": ([_P, C.c_uint32, C.c_uint32, _P, _P], None),
        "ora_volumetrace_f32": ([_P, _P, C.c_uint32, C.c_uint32, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                 C.c_int, _P, C.c_int, _P], None),
        "ora_gdpt_frames": ([_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _P, _P, _P, _P, _P,
                             C.c_int], None),
        "ora_gdpt_reconstruct": ([_P, _P, _P, _P, _P, C.c_uint32, C.c_uint32, _P, _P, _P, _P, C.c_int], None),
        "ora_raytrace": ([_P, _P, C.c_uint32, C.c_uint32, _P, C.c_int], None),
        "ora_scene_set_texture": ([_P, _P, C.c_uint32, C.c_uint32], None),
        "ora_scene_set_object_texture": ([_P, C.c_int, _P, _P, _P], None),
        "ora_pathtrace_phys": ([_P, C.c_int, _P, C.c_uint32, C.c_uint32, _P, C.c_uint32, C.c_uint32, C.c_uint32,
                                C.c_uint32, C.c_int, C.c_int, _P, C.c_int, _P], None),
        "ora_volumetrace_phys_f32": ([_P, _P, C.c_uint32, C.c_uint32, _P, C.c_uint32, C.c_uint32, C.c_uint32,
                                      C.c_uint32, C.c_int, _P, C.c_int, _P], None),
        "ora_medium_forward": ([_P, C.c_int, _P, _P, _P, _P, _P, C.c_uint32, C.c_uint32, _P, C.c_uint32, C.c_uint32,
                                C.c_uint32, C.c_uint32, _P, C.c_int], None),
        "ora_medium_backward": ([_P, C.c_int, _P, _P, _P, _P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32,
                                 C.c_uint32, _P, _P, _P, C.c_int], None),
    }
    for k, (a, r) in sig.items():
        f = getattr(lib, k)
        f.argtypes, f.restype = a, r
    return lib


def _load_ref() -> Optional[C.CDLL]:
    if not os.path.exists(REF_HOST_LIB):
        return None
    lib = C.CDLL(REF_HOST_LIB)
    sig = {
        "ref_scene_new": ([], _P), "ref_scene_free": ([_P], None),
        "ref_scene_add_object": ([_P, C.c_int, _P, C.c_float, _P, _P, C.c_int, _P], None),
        "ref_scene_add_light": ([_P, _P], None), "ref_scene_set_env": ([_P, _P, C.c_uint32, C.c_uint32], None),
        "ref_scene_finalize": ([_P], None),
        "ref_trace": ([_P, C.c_int, _P, _P, _P, _P, _P, _P], None),
        "ref_visible": ([_P, C.c_int, _P, _P, _P, _P], None),
        "ref_pathtrace": ([_P, _P, C.c_uint32, C.c_uint32, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int,
                           _P, C.c_int, _P], None),
        "ref_tea4": ([C.c_uint32, C.c_uint32], C.c_uint32), "ref_rnd_stream": ([C.c_uint32, C.c_int, _P, _P], None),
        "ref_sample_direction": ([_P, C.c_uint32, _P, _P, _P, _P], None), "ref_brdf": ([_P, _P, _P, _P, _P], None),
        "ref_light_sample": ([_P, C.c_uint32, _P, _P, _P, _P, _P], None),
        "ref_volumetrace": ([_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, _P], None),
        "ref_scene_set_volume": ([_P, _P, _P, C.c_float], None),
        "ref_raytrace": ([_P, _P, C.c_uint32, C.c_uint32, _P], None),
        "ref_gdpt_frames": ([_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _P, _P, _P, _P,
                             _P], None),
    }
    for k, (a, r) in sig.items():
        f = getattr(lib, k)
        f.argtypes, f.restype = a, r
    return lib


_oracle = None
_ref = None


def oracle_lib() -> C.CDLL:
    global _oracle
    if _oracle is None:
        _oracle = _load_oracle()
    return _oracle


def ref_lib() -> Optional[C.CDLL]:
    global _ref
    if _ref is None:
        _ref = _load_ref()
    return _ref


class CheckerScene:
    """A scene inside the oracle ("oracle") or the reference host build ("ref")."""

    def __init__(self, desc, kind: str = "oracle"):
        self.kind = kind
        self.lib = oracle_lib() if kind == "oracle" else ref_lib()
        if self.lib is None:
            raise RuntimeError("reference host build not available")
        self._keep = []
        pre = "ora_" if kind == "oracle" else "ref_"
        self.h = self.lib.ora_scene_new(32) if kind == "oracle" else self.lib.ref_scene_new()
        add = getattr(self.lib, pre + "scene_add_object")
        for typ, geo, radius, mat, tris, box in desc.flat():
            self._keep += [geo, mat, tris, box]
            add(self.h, int(typ), _ptr(geo), float(radius), _ptr(mat), _ptr(tris),
                0 if tris is None else len(tris), _ptr(box))
        for l in desc.lights:
            lf = l.flat()
            self._keep.append(lf)
            getattr(self.lib, pre + "scene_add_light")(self.h, _ptr(lf))
        if desc.env is not None:
            env = np.ascontiguousarray(desc.env, dtype=np.float32)
            self._keep.append(env)
            getattr(self.lib, pre + "scene_set_env")(self.h, _ptr(env), env.shape[1], env.shape[0])
        if getattr(desc, "texture", None) is not None:
            if kind != "oracle":
                raise RuntimeError("the reference has no albedo textures")
            tex = np.ascontiguousarray(desc.texture, dtype=np.float32)
            self._keep.append(tex)
            self.lib.ora_scene_set_texture(self.h, _ptr(tex), tex.shape[1], tex.shape[0])
            for i, o in enumerate(desc.objects):
                if getattr(o, "tex_frame", None) is not None:
                    fr = [np.ascontiguousarray(x, np.float32) for x in o.tex_frame]
                    self._keep += fr
                    self.lib.ora_scene_set_object_texture(self.h, i, _ptr(fr[0]), _ptr(fr[1]), _ptr(fr[2]))
        if desc.volume is not None:
            s = np.asarray(desc.volume[0], np.float32)
            a = np.asarray(desc.volume[1], np.float32)
            self._keep += [s, a]
            getattr(self.lib, pre + "scene_set_volume")(self.h, _ptr(s), _ptr(a), float(desc.volume[2]))
        getattr(self.lib, pre + "scene_finalize")(self.h)

    def trace(self, o: np.ndarray, d: np.ndarray, threads: int = 0):
        o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
        n = len(o)
        t = np.empty(n, np.float32)
        obj = np.empty(n, np.int32)
        tri = np.full(n, -1, np.int32)
        P = np.empty((n, 3), np.float32)
        Nn = np.empty((n, 3), np.float32)
        if self.kind == "oracle":
            self.lib.ora_trace(self.h, n, _ptr(o), _ptr(d), _ptr(t), _ptr(obj), _ptr(tri), _ptr(P), _ptr(Nn), threads)
        else:
            self.lib.ref_trace(self.h, n, _ptr(o), _ptr(d), _ptr(t), _ptr(obj), _ptr(P), _ptr(Nn))
        return t, obj, tri, P, Nn

    def visible(self, o, d, dist, threads: int = 0) -> np.ndarray:
        o = np.ascontiguousarray(o, np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(d, np.float32).reshape(-1, 3)
        dist = np.ascontiguousarray(dist, np.float32).reshape(-1)
        vis = np.empty(len(o), np.int32)
        if self.kind == "oracle":
            self.lib.ora_visible(self.h, len(o), _ptr(o), _ptr(d), _ptr(dist), _ptr(vis), threads)
        else:
            self.lib.ref_visible(self.h, len(o), _ptr(o), _ptr(d), _ptr(dist), _ptr(vis))
        return vis.astype(bool)

    def pathtrace(self, cam: np.ndarray, w: int, h: int, frame0: int, nframes: int, max_depth: int, rr: bool = False,
                  pixels: Optional[np.ndarray] = None, img: Optional[np.ndarray] = None, threads: int = 0,
                  precision: int = 32):
        """Running-mean image after frames [frame0, frame0 + nframes).  Returns (img, (ext_rays, shadow_rays))."""
        cam = np.ascontiguousarray(cam, np.float32)
        npix = w * h if pixels is None else len(pixels)
        dtype = np.float64 if precision == 64 else np.float32
        if img is None:
            img = np.zeros((npix, 3), dtype)
        img = np.ascontiguousarray(img, dtype)
        px = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
        counts = np.zeros(2, np.uint64)
        if self.kind == "oracle":
            fn = self.lib.ora_pathtrace_f64 if precision == 64 else self.lib.ora_pathtrace_f32
            fn(self.h, _ptr(cam), w, h, _ptr(px), npix, frame0, nframes, max_depth, int(rr), _ptr(img), threads,
               _ptr(counts))
        else:
            self.lib.ref_pathtrace(self.h, _ptr(cam), w, h, _ptr(px), npix, frame0, nframes, max_depth, int(rr),
                                   _ptr(img), threads if threads > 0 else (os.cpu_count() or 1), _ptr(counts))
        return img, (int(counts[0]), int(counts[1]))

    def pathtrace_cached(self, cam, w: int, h: int, frame0: int, nframes: int, max_depth: int, cache_depth: int,
                         value, img: Optional[np.ndarray] = None, threads: int = 0, specular: bool = False):
        """The cached path tracer's running mean with a cache that answers
        `value` (RGB) everywhere (oracle only, float)."""
        cam = np.ascontiguousarray(cam, np.float32)
        img = np.zeros((w * h, 3), np.float32) if img is None else np.ascontiguousarray(img, np.float32).copy()
        v = np.ascontiguousarray(value, np.float32).reshape(3)
        self.lib.ora_pathtrace_cached_f32(self.h, _ptr(cam), w, h, frame0, nframes, max_depth, cache_depth, _ptr(v),
                                          1 if specular else 0, _ptr(img), threads)
        return img

    def pathtrace_physical(self, cam, w: int, h: int, frame0: int, nframes: int, max_depth: int, mode: str = "mis",
                           rr: bool = False, pixels: Optional[np.ndarray] = None, threads: int = 0,
                           precision: int = 32) -> np.ndarray:
        """Running mean of the physical estimators (oracle only): "mis" (what
        CUPBR_ESTIMATOR_PHYSICAL computes), "nee" (environment by light
        sampling only) or "bsdf" (environment by BSDF sampling only)."""
        modes = {"mis": 1, "nee": 2, "bsdf": 3}
        cam = np.ascontiguousarray(cam, np.float32)
        npix = w * h if pixels is None else len(pixels)
        img = np.zeros((npix, 3), np.float64 if precision == 64 else np.float32)
        px = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
        self.lib.ora_pathtrace_phys(self.h, 64 if precision == 64 else 32, _ptr(cam), w, h, _ptr(px), npix, frame0,
                                    nframes, max_depth, int(rr), modes[mode], _ptr(img), threads, None)
        return img

    def volumetrace(self, cam, w: int, h: int, frame0: int, nframes: int, max_depth: int, rr: bool = False,
                    img: Optional[np.ndarray] = None, threads: int = 0, physical: bool = False):
        """VOLUME method running mean (VolumeRenderer.cu:214-310); physical:
        the scene medium's light term with its phase value (oracle only)."""
        cam = np.ascontiguousarray(cam, np.float32)
        img = np.zeros((w * h, 3), np.float32) if img is None else np.ascontiguousarray(img, np.float32).copy()
        if self.kind == "oracle":
            fn = self.lib.ora_volumetrace_phys_f32 if physical else self.lib.ora_volumetrace_f32
            fn(self.h, _ptr(cam), w, h, None, w * h, frame0, nframes, max_depth, int(rr), _ptr(img), threads, None)
        else:
            self.lib.ref_volumetrace(self.h, _ptr(cam), w, h, frame0, nframes, max_depth, int(rr), _ptr(img))
        return img

    def raytrace(self, cam, w: int, h: int, threads: int = 0):
        """RAYTRACER method image (RayTracer.cu:11-54)."""
        cam = np.ascontiguousarray(cam, np.float32)
        img = np.zeros((w * h, 3), np.float32)
        if self.kind == "oracle":
            self.lib.ora_raytrace(self.h, _ptr(cam), w, h, _ptr(img), threads)
        else:
            self.lib.ref_raytrace(self.h, _ptr(cam), w, h, _ptr(img))
        return img

    def gdpt(self, cam, w: int, h: int, frame0: int, nframes: int, max_depth: int, imgs=None, threads: int = 0):
        """GRADIENTDOMAIN frames: returns the running means [base, gxf, gxb, gyf, gyb]."""
        cam = np.ascontiguousarray(cam, np.float32)
        imgs = [np.zeros((w * h, 3), np.float32) for _ in range(5)] if imgs is None else \
            [np.ascontiguousarray(a, np.float32).copy() for a in imgs]
        p = [_ptr(a) for a in imgs]
        if self.kind == "oracle":
            self.lib.ora_gdpt_frames(self.h, _ptr(cam), w, h, frame0, nframes, max_depth, *p, threads)
        else:
            self.lib.ref_gdpt_frames(self.h, _ptr(cam), w, h, frame0, nframes, max_depth, *p)
        return imgs

    # -- density-grid medium (oracle only) --------------------------------
    @staticmethod
    def _medium_args(grid, box, majorant, albedo, g, q, precision):
        dt = np.float64 if precision == 64 else np.float32
        dens = np.ascontiguousarray(grid, dt)
        dims = np.array([dens.shape[2], dens.shape[1], dens.shape[0]], np.uint32)
        boxf = np.ascontiguousarray(np.asarray(box, np.float32).reshape(6))
        mp = np.array([majorant, albedo, g, q], np.float32)
        return dt, dens, dims, boxf, mp

    def medium_forward(self, grid, box, majorant, albedo, g, q, cam, w, h, spp, frame0, max_depth,
                       pixels=None, precision=32, threads=0):
        """Grid-medium image (npix, 3): mean of spp samples per pixel."""
        assert self.kind == "oracle"
        dt, dens, dims, boxf, mp = self._medium_args(grid, box, majorant, albedo, g, q, precision)
        cam = np.ascontiguousarray(cam, np.float32)
        px = None if pixels is None else np.ascontiguousarray(pixels, np.uint32)
        n = w * h if px is None else len(px)
        img = np.zeros((n, 3), dt)
        self.lib.ora_medium_forward(self.h, precision, _ptr(dims), _ptr(boxf), _ptr(mp), _ptr(dens), _ptr(cam), w, h,
                                    _ptr(px), n, spp, frame0, max_depth, _ptr(img), threads)
        return img

    def medium_backward(self, grid, box, majorant, albedo, g, q, cam, w, h, spp, frame0, max_depth, grad_img,
                        n_params, precision=32, threads=0):
        """(dLoss/d grid, dLoss/d params) for dLoss/d image = grad_img."""
        assert self.kind == "oracle"
        dt, dens, dims, boxf, mp = self._medium_args(grid, box, majorant, albedo, g, q, precision)
        cam = np.ascontiguousarray(cam, np.float32)
        gi = np.ascontiguousarray(grad_img, dt).reshape(-1)
        gg = np.zeros(dens.size, dt)
        gp = np.zeros(n_params, dt)
        self.lib.ora_medium_backward(self.h, precision, _ptr(dims), _ptr(boxf), _ptr(mp), _ptr(dens), _ptr(cam), w,
                                     h, spp, frame0, max_depth, _ptr(gi), _ptr(gg), _ptr(gp), threads)
        return gg.reshape(dens.shape), gp

    def __del__(self):
        try:
            if self.kind == "oracle":
                self.lib.ora_scene_free(self.h)
        except Exception:
            pass


def gdpt_reconstruct(imgs, w: int, h: int, temp: Optional[np.ndarray] = None, iterations: int = 50):
    """init_kernel + optimization passes: returns (output, gradient_x, gradient_y)."""
    a = [np.ascontiguousarray(x, np.float32) for x in imgs]
    temp = np.zeros((w * h, 3), np.float32) if temp is None else np.ascontiguousarray(temp, np.float32).copy()
    out = np.zeros((w * h, 3), np.float32)
    gx = np.zeros((w * h, 3), np.float32)
    gy = np.zeros((w * h, 3), np.float32)
    oracle_lib().ora_gdpt_reconstruct(*[_ptr(x) for x in a], w, h, _ptr(temp), _ptr(out), _ptr(gx), _ptr(gy),
                                      iterations)
    return out, gx, gy


def tonemap(hdr: np.ndarray, type_: int, exposure: float = 1.0) -> np.ndarray:
    hdr = np.ascontiguousarray(hdr, np.float32)
    n = hdr.size // 3
    out = np.empty(n * 4, np.uint8)
    oracle_lib().ora_tonemap(_ptr(hdr), n, int(type_), float(exposure), _ptr(out))
    return out.reshape(hdr.shape[:-1] + (4,))


def bloom(hdr: np.ndarray, threshold) -> np.ndarray:
    hdr = np.ascontiguousarray(hdr, np.float32)
    h, w, _ = hdr.shape
    th = np.asarray(threshold, np.float32)
    out = np.empty_like(hdr)
    oracle_lib().ora_bloom(_ptr(hdr), w, h, _ptr(th), _ptr(out))
    return out


# ------------------------------------------------------ reference CUDA build
REF_CUDA_LIB = os.path.join(HERE, "_ref", "libref_cuda.so")
_refcu = None


def ref_cuda_lib() -> Optional[C.CDLL]:
    """The reference's own CUDA path built for sm_100a (oracle/ref_cuda.cu)."""
    global _refcu
    if _refcu is None and os.path.exists(REF_CUDA_LIB):
        lib = C.CDLL(REF_CUDA_LIB)
        sig = {
            "refcu_scene_new": ([], _P),
            "refcu_scene_add_object": ([_P, C.c_int, _P, C.c_float, _P, _P, C.c_int, _P], None),
            "refcu_scene_add_light": ([_P, _P], None),
            "refcu_scene_set_env": ([_P, _P, C.c_uint32, C.c_uint32], None),
            "refcu_scene_finalize": ([_P], C.c_int),
            "refcu_pathtrace": ([_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, _P, _P],
                                C.c_int),
            "refcu_bloom": ([_P, C.c_uint32, C.c_uint32, _P, _P], C.c_int),
            "refcu_tonemap": ([_P, C.c_uint32, C.c_uint32, C.c_int, C.c_float, _P], C.c_int),
            "refcu_scene_set_volume": ([_P, _P, _P, C.c_float], None),
            "refcu_volumetrace": ([_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_int, _P,
                                   _P], C.c_int),
            "refcu_gradientdomain": ([_P, _P, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, C.c_uint32, _P, _P],
                                     C.c_int),
            "refcu_raytrace": ([_P, _P, C.c_uint32, C.c_uint32, _P], C.c_int),
        }
        for k, (a, r) in sig.items():
            f = getattr(lib, k)
            f.argtypes, f.restype = a, r
        _refcu = lib
    return _refcu


class RefCudaScene:
    """A scene inside the reference's own CUDA build (device resident)."""

    def __init__(self, desc):
        self.lib = ref_cuda_lib()
        if self.lib is None:
            raise RuntimeError("reference CUDA build not available")
        self._keep = []
        self.h = self.lib.refcu_scene_new()
        for typ, geo, radius, mat, tris, box in desc.flat():
            self._keep += [geo, mat, tris, box]
            self.lib.refcu_scene_add_object(self.h, int(typ), _ptr(geo), float(radius), _ptr(mat), _ptr(tris),
                                            0 if tris is None else len(tris), _ptr(box))
        for l in desc.lights:
            lf = l.flat()
            self._keep.append(lf)
            self.lib.refcu_scene_add_light(self.h, _ptr(lf))
        if desc.env is not None:
            env = np.ascontiguousarray(desc.env, dtype=np.float32)
            self._keep.append(env)
            self.lib.refcu_scene_set_env(self.h, _ptr(env), env.shape[1], env.shape[0])
        # the reference has no albedo textures: a textured description is
        # rendered with its materials' own albedos (throughput comparisons only)
        if desc.volume is not None:
            s = np.asarray(desc.volume[0], np.float32)
            a = np.asarray(desc.volume[1], np.float32)
            self._keep += [s, a]
            self.lib.refcu_scene_set_volume(self.h, _ptr(s), _ptr(a), float(desc.volume[2]))
        rc = self.lib.refcu_scene_finalize(self.h)
        if rc != 0:
            raise RuntimeError(f"reference scene upload failed: cuda error {rc}")

    def pathtrace(self, cam, w: int, h: int, frame0: int, nframes: int, max_depth: int, rr: bool = False, img=None):
        """Returns (running-mean image (h*w, 3), device ms of the render calls)."""
        cam = np.ascontiguousarray(cam, np.float32)
        img = np.zeros((w * h, 3), np.float32) if img is None else np.ascontiguousarray(img, np.float32).copy()
        ms = np.zeros(1, np.float32)
        rc = self.lib.refcu_pathtrace(self.h, _ptr(cam), w, h, frame0, nframes, max_depth, int(rr), _ptr(img),
                                      _ptr(ms))
        if rc != 0:
            raise RuntimeError(f"reference pathtracing failed: cuda error {rc}")
        return img, float(ms[0])

    def volumetrace(self, cam, w, h, frame0, nframes, max_depth, rr=False):
        cam = np.ascontiguousarray(cam, np.float32)
        img = np.zeros((w * h, 3), np.float32)
        ms = np.zeros(1, np.float32)
        rc = self.lib.refcu_volumetrace(self.h, _ptr(cam), w, h, frame0, nframes, max_depth, int(rr), _ptr(img),
                                        _ptr(ms))
        if rc != 0:
            raise RuntimeError(f"reference volumetracing failed: cuda error {rc}")
        return img, float(ms[0])

    def gradientdomain(self, cam, w, h, frame0, nframes, max_depth):
        """Returns (dict of the nine buffers, ms)."""
        cam = np.ascontiguousarray(cam, np.float32)
        out = np.zeros((9, w * h, 3), np.float32)
        ms = np.zeros(1, np.float32)
        rc = self.lib.refcu_gradientdomain(self.h, _ptr(cam), w, h, frame0, nframes, max_depth, _ptr(out), _ptr(ms))
        if rc != 0:
            raise RuntimeError(f"reference gradientdomain failed: cuda error {rc}")
        keys = ("output", "gradient_x", "gradient_y", "base", "gxf", "gxb", "gyf", "gyb", "temp")
        return dict(zip(keys, out)), float(ms[0])

    def raytrace(self, cam, w, h):
        cam = np.ascontiguousarray(cam, np.float32)
        img = np.zeros((w * h, 3), np.float32)
        rc = self.lib.refcu_raytrace(self.h, _ptr(cam), w, h, _ptr(img))
        if rc != 0:
            raise RuntimeError(f"reference raytracing failed: cuda error {rc}")
        return img


def ref_cuda_bloom(hdr: np.ndarray, threshold) -> np.ndarray:
    hdr = np.ascontiguousarray(hdr, np.float32)
    h, w, _ = hdr.shape
    th = np.asarray(threshold, np.float32)
    out = np.empty_like(hdr)
    rc = ref_cuda_lib().refcu_bloom(_ptr(hdr), w, h, _ptr(th), _ptr(out))
    if rc != 0:
        raise RuntimeError(f"reference bloom failed: {rc}")
    return out


def ref_cuda_post_timed(hdr: np.ndarray, threshold, type_: int = 0, exposure: float = 1.0, iters: int = 5):
    """The reference's bloom and tone map on the device, timed: (ms per
    bloom, ms per tone map)."""
    hdr = np.ascontiguousarray(hdr, np.float32)
    h, w, _ = hdr.shape
    th = np.asarray(threshold, np.float32)
    ms = np.zeros(2, np.float32)
    lib = ref_cuda_lib()
    lib.refcu_post_timed.argtypes = [_P, C.c_uint32, C.c_uint32, _P, C.c_int, C.c_float, C.c_uint32, _P]
    lib.refcu_post_timed.restype = C.c_int
    rc = lib.refcu_post_timed(_ptr(hdr), w, h, _ptr(th), int(type_), float(exposure), int(iters), _ptr(ms))
    if rc != 0:
        raise RuntimeError(f"reference post-processing failed: {rc}")
    return float(ms[0]), float(ms[1])


def ref_cuda_tonemap(hdr: np.ndarray, type_: int, exposure: float = 1.0) -> np.ndarray:
    hdr = np.ascontiguousarray(hdr, np.float32)
    h, w, _ = hdr.shape
    out = np.empty((h, w, 4), np.uint8)
    rc = ref_cuda_lib().refcu_tonemap(_ptr(hdr), w, h, int(type_), float(exposure), _ptr(out))
    if rc != 0:
        raise RuntimeError(f"reference tone map failed: {rc}")
    return out

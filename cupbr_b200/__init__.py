"""cupbr-b200: B200-native rendering hot path of cupbr behind its own API.

Python mirror of cupbr's renderer surface over the C ABI (include/cupbr_c.h):
  PBRenderer / RenderingMethod   lib/include/Renderer/PBRenderer.h:14-116
  ToneMapper / ToneMappingType   lib/include/Renderer/ToneMapper.h:14-80
  PostProcessor                  lib/include/PostProcessing/PostProcessor.h:12-52
  SceneLoader.load_from_file     lib/include/Scene/SceneLoader.h:8-22
  Camera(width, height)          lib/src/DataStructure/Camera.cpp:6-11
Methods keep the reference's names (snake_case) and semantics; precondition
failures raise CupbrError instead of printing to std::cerr.
"""
from __future__ import annotations

import ctypes as C
import enum
from typing import Optional

import numpy as np

from . import _native as N
from ._native import CupbrError
from . import scenes
from .scenes import SceneDesc, MaterialDesc, LightDesc, ObjectDesc

__all__ = ["RenderingMethod", "ToneMappingType", "Camera", "Scene", "SceneLoader", "PBRenderer", "ToneMapper", "Batch",
           "PostProcessor", "DeviceImage", "CupbrError", "SceneDesc", "MaterialDesc", "LightDesc", "ObjectDesc",
           "scenes", "threshold_curve", "library_path"]

library_path = N.LIB_PATH


class RenderingMethod(enum.IntEnum):
    RAYTRACER = 0
    WHITTED = 1
    PATHTRACER = 2
    METROPOLIS = 3
    GRADIENTDOMAIN = 4
    VOLUME = 5


class ToneMappingType(enum.IntEnum):
    REINHARD = 0
    GAMMA = 1


def threshold_curve(threshold: float = 1.0, knee: float = 1.0) -> tuple:
    """Interactor::compute_threshold (Interactor.cpp:436-440)."""
    return (np.float32(threshold), np.float32(knee - threshold), np.float32(2.0 * knee), np.float32(0.25 / knee))


def _stream_ptr(stream) -> Optional[int]:
    if stream is None:
        return None
    if isinstance(stream, int):
        return stream
    return int(stream.cuda_stream)  # torch.cuda.Stream


class DeviceImage:
    """A device buffer owned by a renderer / tone mapper / post processor.
    Exposes __cuda_array_interface__ so torch.as_tensor(img, device="cuda")
    views it without a copy."""

    def __init__(self, ptr: int, width: int, height: int, channels: int, dtype, owner=None):
        self.ptr, self.width, self.height, self.channels = int(ptr or 0), width, height, channels
        self.dtype = np.dtype(dtype)
        self._owner = owner

    @property
    def shape(self):
        return (self.height, self.width, self.channels)

    @property
    def nbytes(self) -> int:
        return self.width * self.height * self.channels * self.dtype.itemsize

    @property
    def __cuda_array_interface__(self):
        return {"shape": self.shape, "typestr": self.dtype.str, "data": (self.ptr, False), "version": 3,
                "strides": None}

    def numpy(self, stream=None) -> np.ndarray:
        out = np.empty(self.shape, dtype=self.dtype)
        N.call("cupbr_memcpy_d2h", out.ctypes.data, self.ptr, self.nbytes, _stream_ptr(stream))
        N.call("cupbr_stream_synchronize", _stream_ptr(stream))
        return out


class Camera:
    """Camera pose (Camera.h:71-75).  Camera(width, height) is the
    reference's default pose: origin, looking +z, x axis scaled by aspect."""

    def __init__(self, width: int = 1, height: int = 1):
        c = N.Camera()
        N.call("cupbr_camera_default", width, height, C.byref(c))
        self._c = c

    @classmethod
    def from_axes(cls, position, x_axis, y_axis, z_axis) -> "Camera":
        cam = cls(1, 1)
        cam._c.position, cam._c.x_axis = N.Vec3.of(position), N.Vec3.of(x_axis)
        cam._c.y_axis, cam._c.z_axis = N.Vec3.of(y_axis), N.Vec3.of(z_axis)
        return cam

    def position(self):
        return self._c.position.tuple()

    def x_axis(self):
        return self._c.x_axis.tuple()

    def y_axis(self):
        return self._c.y_axis.tuple()

    def z_axis(self):
        return self._c.z_axis.tuple()

    def moved(self) -> bool:
        return bool(self._c.moved)

    def set_moved(self, moved: bool) -> None:
        self._c.moved = 1 if moved else 0

    def flat(self) -> np.ndarray:
        """12 floats (position, x, y, z axes) for the CPU checkers."""
        return np.array([*self.position(), *self.x_axis(), *self.y_axis(), *self.z_axis()], dtype=np.float32)


def _mat(m: MaterialDesc) -> N.Material:
    return N.Material(int(m.type), N.Vec3.of(m.albedo_e), N.Vec3.of(m.albedo_d), N.Vec3.of(m.albedo_s),
                      float(m.shininess), float(m.roughness), float(m.eta), N.Vec3.of(m.sigma_s),
                      N.Vec3.of(m.sigma_a), float(m.g), int(m.interface_glass))


def _bvh(params: Optional[dict]):
    if params is None:
        return None
    builder = params.get("builder", "device")
    if builder not in ("host", "device"):
        raise ValueError(f"bvh builder must be 'host' or 'device', not {builder!r}")
    p = N.BvhParams(int(params.get("max_leaf_size", 4)), float(params.get("traversal_cost", 2.0)),
                    int(params.get("top_bfs_levels", 4)), 1 if builder == "host" else 0)
    return C.byref(p)


class Scene:
    """A committed, GPU-resident scene (cupbr_scene_t)."""

    def __init__(self, handle: int):
        self._h = C.c_void_p(handle)

    @classmethod
    def from_desc(cls, desc: SceneDesc, bvh_params: Optional[dict] = None) -> "Scene":
        h = C.c_void_p()
        N.call("cupbr_scene_create", C.byref(h))
        s = cls(h.value)
        try:
            for o in desc.objects:
                m = C.byref(_mat(o.material))
                if o.type == scenes.SPHERE:
                    N.call("cupbr_scene_add_sphere", s._h, N.Vec3.of(o.p0), float(o.radius), m, None)
                elif o.type == scenes.PLANE:
                    N.call("cupbr_scene_add_plane", s._h, N.Vec3.of(o.p0), N.Vec3.of(o.p1), m, None)
                elif o.type == scenes.QUAD:
                    N.call("cupbr_scene_add_quad", s._h, N.Vec3.of(o.p0), N.Vec3.of(o.p1), N.Vec3.of(o.p2),
                           N.Vec3.of(o.p3), m, None)
                elif o.type == scenes.TRIANGLE:
                    v = np.asarray(o.vertices, dtype=np.float32).reshape(3, 3)
                    N.call("cupbr_scene_add_triangle", s._h, N.Vec3.of(v[0]), N.Vec3.of(v[1]), N.Vec3.of(v[2]), m,
                           None)
                else:
                    v = np.ascontiguousarray(o.vertices, dtype=np.float32)
                    idx = np.ascontiguousarray(o.indices, dtype=np.uint32)
                    N.call("cupbr_scene_add_mesh", s._h, v.ctypes.data, len(v), idx.ctypes.data, len(idx),
                           N.Vec3.of(o.position), N.Vec3.of(o.scale), m, None)
            for l in desc.lights:
                li = N.Light(int(l.type), N.Vec3.of(l.position), N.Vec3.of(l.intensity), N.Vec3.of(l.radiance),
                             N.Vec3.of(l.half_extend1), N.Vec3.of(l.half_extend2))
                N.call("cupbr_scene_add_light", s._h, C.byref(li))
            if desc.volume is not None:
                ss, sa, g = desc.volume
                N.call("cupbr_scene_set_volume", s._h, N.Vec3.of(ss), N.Vec3.of(sa), float(g))
            if desc.env is not None:
                env = np.ascontiguousarray(desc.env, dtype=np.float32)
                N.call("cupbr_scene_set_environment", s._h, env.ctypes.data, env.shape[1], env.shape[0])
            if desc.camera is not None:
                s.set_camera(*desc.camera)
            if desc.texture is not None:
                tex = np.ascontiguousarray(desc.texture, dtype=np.float32)
                N.call("cupbr_scene_set_albedo_texture", s._h, tex.ctypes.data, tex.shape[1], tex.shape[0])
                for i, o in enumerate(desc.objects):
                    if o.tex_frame is not None:
                        org, u, v = o.tex_frame
                        N.call("cupbr_scene_set_object_texture", s._h, i, N.Vec3.of(org), N.Vec3.of(u), N.Vec3.of(v))
            N.call("cupbr_scene_commit", s._h, _bvh(bvh_params))
        except Exception:
            s.destroy()
            raise
        return s

    def commit(self, bvh_params: Optional[dict] = None) -> None:
        N.call("cupbr_scene_commit", self._h, _bvh(bvh_params))

    def destroy(self) -> None:
        if self._h:
            N.call("cupbr_scene_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    def albedo_texture_or_none(self) -> Optional[DeviceImage]:
        try:
            return self.albedo_texture()
        except CupbrError:
            return None

    def albedo_texture(self) -> DeviceImage:
        """The committed albedo texture on the device: height x width x 4
        floats (RGB + unused), writable (cupbr_scene_get_albedo_texture)."""
        p, w, h = C.c_void_p(), C.c_uint32(), C.c_uint32()
        N.call("cupbr_scene_get_albedo_texture", self._h, C.byref(p), C.byref(w), C.byref(h))
        if not p.value:
            raise CupbrError(-4, "scene has no albedo texture")
        return DeviceImage(p.value, w.value, h.value, 4, np.float32, owner=self)

    def info(self) -> dict:
        i = N.SceneInfo()
        N.call("cupbr_scene_get_info", self._h, C.byref(i))
        return {k: getattr(i, k) for k, _ in N.SceneInfo._fields_}

    def object(self, index: int) -> N.ObjectDesc:
        o = N.ObjectDesc()
        N.call("cupbr_scene_get_object", self._h, index, C.byref(o))
        return o

    def object_triangles(self, index: int) -> np.ndarray:
        n = self.object(index).triangle_count
        out = np.empty((n, 9), dtype=np.float32)
        N.call("cupbr_scene_get_triangles", self._h, index, out.ctypes.data, n)
        return out

    def bvh_nodes(self) -> np.ndarray:
        """The BVH the traversal kernels read: (nodes, 32) float32, per node
        the x / y / z bounds of its four children, then their references
        (int32 bits: inner node index, or ~(slot << 3 | count - 1) for a leaf)."""
        n = C.c_uint32()
        N.call("cupbr_scene_get_bvh", self._h, None, 0, C.byref(n))
        out = np.empty((n.value, 32), dtype=np.float32)
        N.call("cupbr_scene_get_bvh", self._h, out.ctypes.data, n.value, C.byref(n))
        return out

    def key_slots(self) -> np.ndarray:
        """Per primitive key: the slot of its primitive in its type's table."""
        n = C.c_uint32()
        N.call("cupbr_scene_get_key_slots", self._h, None, 0, C.byref(n))
        out = np.empty(n.value, dtype=np.uint32)
        N.call("cupbr_scene_get_key_slots", self._h, out.ctypes.data, n.value, C.byref(n))
        return out

    def camera(self, width: int, height: int) -> "Camera":
        """The scene file's <camera> pose for a width x height view (the
        default Camera(width, height) when the file has none)."""
        cam = Camera(width, height)
        N.call("cupbr_scene_get_camera", self._h, width, height, C.byref(cam._c))
        return cam

    def set_camera(self, position, yaw: float, pitch: float) -> None:
        N.call("cupbr_scene_set_camera", self._h, N.Vec3.of(position), float(yaw), float(pitch))

    def pick(self, camera: "Camera", x: int, y: int, width: int, height: int):
        """Interaction::pickMouse (MousePicker.cu:55-72): (scene index, material)
        of the object seen through pixel (x, y), or None on a miss."""
        m = N.Material()
        idx = C.c_int32(-1)
        N.call("cupbr_scene_pick", self._h, C.byref(camera._c), x, y, width, height, C.byref(m), C.byref(idx))
        return None if idx.value < 0 else (idx.value, m)

    def update_material(self, index: int, material: MaterialDesc) -> None:
        """Interaction::updateMaterial (MousePicker.cu:74-81)."""
        N.call("cupbr_scene_update_material", self._h, int(index), C.byref(_mat(material)))

    def light(self, index: int) -> N.Light:
        l = N.Light()
        N.call("cupbr_scene_get_light", self._h, index, C.byref(l))
        return l

    def trace(self, origins: np.ndarray, directions: np.ndarray):
        """Closest hit for host rays: (depth, object id, triangle index)."""
        o = np.ascontiguousarray(origins, dtype=np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, dtype=np.float32).reshape(-1, 3)
        n = len(o)
        t = np.empty(n, np.float32)
        obj = np.empty(n, np.int32)
        tri = np.empty(n, np.int32)
        N.call("cupbr_scene_trace", self._h, n, o.ctypes.data, d.ctypes.data, t.ctypes.data, obj.ctypes.data,
               tri.ctypes.data)
        return t, obj, tri

    def visible(self, origins: np.ndarray, directions: np.ndarray, light_distance: np.ndarray) -> np.ndarray:
        o = np.ascontiguousarray(origins, dtype=np.float32).reshape(-1, 3)
        d = np.ascontiguousarray(directions, dtype=np.float32).reshape(-1, 3)
        dist = np.ascontiguousarray(light_distance, dtype=np.float32).reshape(-1)
        vis = np.empty(len(o), np.int32)
        N.call("cupbr_scene_visible", self._h, len(o), o.ctypes.data, d.ctypes.data, dist.ctypes.data,
               vis.ctypes.data)
        return vis.astype(bool)


class SceneLoader:
    """SceneLoader::loadFromFile / destroyScene (SceneLoader.h:8-22)."""

    @staticmethod
    def load_from_file(path: str, bvh_params: Optional[dict] = None) -> Scene:
        h = C.c_void_p()
        N.call("cupbr_scene_load_xml_ex", path.encode(), _bvh(bvh_params), C.byref(h))
        return Scene(h.value)

    @staticmethod
    def parse_file(path: str) -> Scene:
        """Parse only (no BVH build, no upload); call Scene.commit() later."""
        h = C.c_void_p()
        N.call("cupbr_scene_parse_xml", path.encode(), C.byref(h))
        return Scene(h.value)

    @staticmethod
    def destroy_scene(scene: Scene) -> None:
        scene.destroy()


class PBRenderer:
    """PBRenderer (lib/include/Renderer/PBRenderer.h:27-116)."""

    def __init__(self, method: RenderingMethod = RenderingMethod.RAYTRACER):
        h = C.c_void_p()
        N.call("cupbr_renderer_create", int(method), C.byref(h))
        self._h = h
        self._scene = None
        self._w = self._h_px = 0

    def __del__(self):
        try:
            if self._h:
                N.call("cupbr_renderer_destroy", self._h)
                self._h = C.c_void_p()
        except Exception:
            pass

    def set_output_size(self, width: int, height: int) -> None:
        N.call("cupbr_renderer_set_output_size", self._h, width, height)
        self._w, self._h_px = width, height

    def register_scene(self, scene: Scene) -> None:
        N.call("cupbr_renderer_register_scene", self._h, scene._h)
        self._scene = scene  # keep it alive

    def set_method(self, method: RenderingMethod) -> None:
        N.call("cupbr_renderer_set_method", self._h, int(method))

    def get_method(self) -> RenderingMethod:
        m = C.c_int32()
        N.call("cupbr_renderer_get_method", self._h, C.byref(m))
        return RenderingMethod(m.value)

    def render(self, camera: Camera) -> None:
        N.call("cupbr_renderer_render", self._h, C.byref(camera._c))

    def render_frames(self, camera: Camera, nframes: int) -> None:
        """nframes render() calls; the path tracer batches frames per wavefront."""
        N.call("cupbr_renderer_render_frames", self._h, C.byref(camera._c), nframes)

    def set_pipelined(self, enable: bool) -> None:
        """render() traces each frame on one of four internal streams in turn
        so later frames overlap the caller's tone mapping / readback of this
        one (and each other's sparse last depths), and render_frames()
        alternates its wavefronts between two of them so they overlap each
        other (same images)."""
        N.call("cupbr_renderer_set_pipelined", self._h, 1 if enable else 0)

    def set_tail_paths(self, paths: int) -> None:
        """Ray queues below `paths` rays (default 2^17 on one stream, off
        when pipelined) finish their paths in one per-path launch (same
        image; 0 = off)."""
        N.call("cupbr_renderer_set_tail_paths", self._h, paths)

    def set_batch_paths(self, paths: int) -> None:
        N.call("cupbr_renderer_set_batch_paths", self._h, paths)

    def get_output_image(self) -> DeviceImage:
        p, w, h = C.c_void_p(), C.c_uint32(), C.c_uint32()
        N.call("cupbr_renderer_get_output", self._h, C.byref(p), C.byref(w), C.byref(h))
        return DeviceImage(p.value, w.value, h.value, 3, np.float32, self)

    def get_gradient_x(self) -> DeviceImage:
        p = C.c_void_p()
        N.call("cupbr_renderer_get_gradient_x", self._h, C.byref(p))
        return DeviceImage(p.value, self._w, self._h_px, 3, np.float32, self)

    def get_gradient_y(self) -> DeviceImage:
        p = C.c_void_p()
        N.call("cupbr_renderer_get_gradient_y", self._h, C.byref(p))
        return DeviceImage(p.value, self._w, self._h_px, 3, np.float32, self)

    def reset(self) -> None:
        N.call("cupbr_renderer_reset", self._h)

    def set_russian_roulette(self, use: bool) -> None:
        N.call("cupbr_renderer_set_russian_roulette", self._h, 1 if use else 0)

    def set_estimator(self, estimator: str) -> None:
        """"reference" (default: the reference's estimator, the parity path)
        or "physical" (environment importance sampling with MIS; the scene
        medium's phase value in VOLUME).  Restarts accumulation
        (cupbr_renderer_set_estimator)."""
        kinds = {"reference": 0, "physical": 1}
        if estimator not in kinds:
            raise ValueError(f"estimator must be one of {sorted(kinds)}")
        N.call("cupbr_renderer_set_estimator", self._h, kinds[estimator])

    def set_persistent(self, enable: bool) -> None:
        """render_frames through one persistent-kernel launch (same image)
        instead of wavefronts (cupbr_renderer_set_persistent)."""
        N.call("cupbr_renderer_set_persistent", self._h, 1 if enable else 0)

    def get_estimator(self) -> str:
        v = C.c_int32()
        N.call("cupbr_renderer_get_estimator", self._h, C.byref(v))
        return ("reference", "physical")[v.value]

    def set_max_trace_depth(self, depth: int) -> None:
        N.call("cupbr_renderer_set_max_trace_depth", self._h, depth)

    def get_max_trace_depth(self) -> int:
        d = C.c_uint32()
        N.call("cupbr_renderer_get_max_trace_depth", self._h, C.byref(d))
        return d.value

    # --- additions: stream, checkpoint/resume, diagnostics
    def set_stream(self, stream) -> None:
        N.call("cupbr_renderer_set_stream", self._h, _stream_ptr(stream))

    def frame_index(self) -> int:
        f = C.c_uint32()
        N.call("cupbr_renderer_get_frame_index", self._h, C.byref(f))
        return f.value

    def set_frame_index(self, f: int) -> None:
        N.call("cupbr_renderer_set_frame_index", self._h, f)

    def error_count(self) -> int:
        c = C.c_uint32()
        N.call("cupbr_renderer_get_error_count", self._h, C.byref(c))
        return c.value

    def set_instrumented(self, on: bool) -> None:
        N.call("cupbr_renderer_set_instrumented", self._h, 1 if on else 0)

    def set_profiling(self, on: bool) -> None:
        N.call("cupbr_renderer_set_profiling", self._h, 1 if on else 0)

    def stage_times(self) -> dict:
        """Summed device ms per stage of the frames rendered while profiling."""
        ms = (C.c_float * 5)()
        frames, launches = C.c_uint32(), C.c_uint32()
        N.call("cupbr_renderer_get_stage_times", self._h, ms, C.byref(frames), C.byref(launches))
        keys = ("camera", "extend", "shade", "connect", "accumulate")
        d = dict(zip(keys, [float(x) for x in ms]))
        d["frames"], d["extend_launches"] = frames.value, launches.value
        return d

    def stats(self) -> dict:
        s = (C.c_uint64 * 6)()
        N.call("cupbr_renderer_get_stats", self._h, s)
        keys = ("ext_nodes", "ext_prims", "shadow_nodes", "shadow_prims", "ext_rays", "shadow_rays")
        return dict(zip(keys, list(s)))


class ToneMapper:
    """ToneMapper (lib/include/Renderer/ToneMapper.h:22-80)."""

    def __init__(self, type: ToneMappingType = ToneMappingType.REINHARD):
        h = C.c_void_p()
        N.call("cupbr_tonemapper_create", int(type), C.byref(h))
        self._h = h
        self._src = None

    def __del__(self):
        try:
            if self._h:
                N.call("cupbr_tonemapper_destroy", self._h)
                self._h = C.c_void_p()
        except Exception:
            pass

    def register_image(self, hdr: DeviceImage) -> None:
        N.call("cupbr_tonemapper_register_image", self._h, hdr.ptr, hdr.width, hdr.height)
        self._src = hdr

    def tone_map(self) -> None:
        N.call("cupbr_tonemapper_tonemap", self._h)

    def get_render_buffer(self) -> DeviceImage:
        p, w, h = C.c_void_p(), C.c_uint32(), C.c_uint32()
        N.call("cupbr_tonemapper_get_render_buffer", self._h, C.byref(p), C.byref(w), C.byref(h))
        return DeviceImage(p.value, w.value, h.value, 4, np.uint8, self)

    def get_type(self) -> ToneMappingType:
        t = C.c_int32()
        N.call("cupbr_tonemapper_get_type", self._h, C.byref(t))
        return ToneMappingType(t.value)

    def set_type(self, type: ToneMappingType) -> None:
        N.call("cupbr_tonemapper_set_type", self._h, int(type))

    def set_exposure(self, exposure: float) -> None:
        N.call("cupbr_tonemapper_set_exposure", self._h, float(exposure))

    def set_stream(self, stream) -> None:
        N.call("cupbr_tonemapper_set_stream", self._h, _stream_ptr(stream))

    def save_to_file(self, path: str) -> None:
        N.call("cupbr_tonemapper_save_to_file", self._h, path.encode())


class PostProcessor:
    """PostProcessor (lib/include/PostProcessing/PostProcessor.h:12-52)."""

    def __init__(self):
        h = C.c_void_p()
        N.call("cupbr_postprocessor_create", C.byref(h))
        self._h = h
        self._src = None

    def __del__(self):
        try:
            if self._h:
                N.call("cupbr_postprocessor_destroy", self._h)
                self._h = C.c_void_p()
        except Exception:
            pass

    def register_image(self, hdr: DeviceImage) -> None:
        N.call("cupbr_postprocessor_register_image", self._h, hdr.ptr, hdr.width, hdr.height)
        self._src = hdr

    def get_post_process_buffer(self) -> DeviceImage:
        p = C.c_void_p()
        N.call("cupbr_postprocessor_get_buffer", self._h, C.byref(p))
        return DeviceImage(p.value, self._src.width, self._src.height, 3, np.float32, self)

    def bloom(self, threshold) -> None:
        th = (C.c_float * 4)(*[float(x) for x in threshold])
        N.call("cupbr_postprocessor_bloom", self._h, th)

    def bloom_tonemap(self, threshold, type: ToneMappingType, exposure: float, rgba: DeviceImage) -> None:
        th = (C.c_float * 4)(*[float(x) for x in threshold])
        N.call("cupbr_postprocessor_bloom_tonemap", self._h, th, int(type), float(exposure), rgba.ptr)

    def set_stream(self, stream) -> None:
        N.call("cupbr_postprocessor_set_stream", self._h, _stream_ptr(stream))


class Batch:
    """Batched multi-view path tracing (cupbr_batch_t): many views of one or
    more scenes in one captured CUDA graph (one persistent-kernel launch by
    default, wavefronts of stage kernels, or the wavefronts' stages in one
    cooperative launch).  `views`
    holds dicts with scene, camera, width, height, spp, frame0 and image
    (a device pointer to width*height RGB floats, the view's running mean).
    A launch gives each view what `spp` PBRenderer.render() calls give it."""

    def __init__(self, views, max_depth: int = 5):
        arr = (N.View * len(views))()
        self._keep = []
        for a, v in zip(arr, views):
            self._keep.append(v["scene"])
            a.scene = v["scene"]._h.value
            a.camera = v["camera"]._c
            a.width, a.height, a.spp = int(v["width"]), int(v["height"]), int(v["spp"])
            a.frame0 = int(v.get("frame0", 0))
            a.device_image = int(v["image"])
        h = C.c_void_p()
        N.call("cupbr_batch_create", arr, len(views), int(max_depth), C.byref(h))
        self._h = h

    def launch(self, stream: Optional[int] = None) -> None:
        N.call("cupbr_batch_launch", self._h, C.c_void_p(stream) if stream else None)

    def advance(self) -> None:
        N.call("cupbr_batch_advance", self._h)

    def set_frame0(self, view: int, frame0: int) -> None:
        N.call("cupbr_batch_set_frame0", self._h, int(view), int(frame0))

    def configure(self, batch_paths: int, trace_share: float = 1.0) -> None:
        N.call("cupbr_batch_configure", self._h, int(batch_paths), float(trace_share))

    def autotune(self, stream: Optional[int] = None, bvh_leaf: bool = False) -> float:
        """Times the candidate configurations (cupbr_batch_autotune_ex) and
        keeps the fastest; bvh_leaf also rebuilds the scenes' BVHs at other
        leaf sizes.  Returns the best median launch time in ms."""
        ms = C.c_float()
        N.call("cupbr_batch_autotune_ex", self._h, C.c_void_p(stream) if stream else None, 1 if bvh_leaf else 0,
               C.byref(ms))
        return ms.value

    MODES = ("wavefront", "persistent", "cooperative")

    def set_mode(self, mode: str, threads_per_block: Optional[int] = None, blocks_per_sm: int = 0,
                 camera_packets: bool = True) -> None:
        """"persistent" (one launch of the per-path persistent kernel),
        "wavefront" (per wavefront, the stage kernels) or "cooperative" (the
        wavefronts' stages in one cooperative launch).  threads_per_block
        defaults to 128 (persistent) or 256 (cooperative, the only shape)."""
        if mode not in self.MODES:
            raise ValueError(f"mode must be one of {sorted(self.MODES)}")
        if threads_per_block is None:
            threads_per_block = 256 if mode == "cooperative" else 128
        N.call("cupbr_batch_set_mode", self._h, self.MODES.index(mode), int(threads_per_block), int(blocks_per_sm),
               1 if camera_packets else 0)

    def mode(self) -> dict:
        m, t, b, p = C.c_int32(), C.c_uint32(), C.c_uint32(), C.c_int32()
        N.call("cupbr_batch_get_mode", self._h, C.byref(m), C.byref(t), C.byref(b), C.byref(p))
        return {"mode": self.MODES[m.value], "threads_per_block": t.value,
                "blocks_per_sm": b.value, "camera_packets": bool(p.value)}

    def error_count(self) -> int:
        v = C.c_uint32()
        N.call("cupbr_batch_get_error_count", self._h, C.byref(v))
        return v.value

    def set_barrier_probe(self, ns: int) -> None:
        """Test hook (cupbr_batch_set_barrier_probe): in the cooperative mode
        one block leaves before the first grid barrier and the others give
        up on it after `ns` nanoseconds (0 = off)."""
        N.call("cupbr_batch_set_barrier_probe", self._h, int(ns))

    def backward(self, grad_images, accumulate: bool = False, stream: Optional[int] = None) -> None:
        """Texture adjoint of the frames of a launch (cupbr_batch_backward):
        grad_images holds one device pointer (or 0) per view to its
        dLoss/dImage (width*height RGB floats)."""
        arr = (C.c_uint64 * len(grad_images))(*[int(p or 0) for p in grad_images])
        N.call("cupbr_batch_backward", self._h, arr, 1 if accumulate else 0, C.c_void_p(stream) if stream else None)

    def texture_gradient(self, scene) -> DeviceImage:
        """The gradient of a scene's albedo texture after backward():
        height x width x 3 floats on the device."""
        p, w, h = C.c_void_p(), C.c_uint32(), C.c_uint32()
        N.call("cupbr_batch_get_texture_gradient", self._h, scene._h, C.byref(p), C.byref(w), C.byref(h))
        if not p.value:
            raise CupbrError(-4, "no texture gradient for this scene (untextured, or backward() not called)")
        return DeviceImage(p.value, w.value, h.value, 3, np.float32, owner=self)

    def info(self) -> dict:
        w, l, bp = C.c_uint32(), C.c_uint32(), C.c_uint32()
        p = C.c_uint64()
        N.call("cupbr_batch_get_info", self._h, C.byref(w), C.byref(p), C.byref(l), C.byref(bp))
        return {"wavefronts": w.value, "paths": p.value, "kernel_launches": l.value, "batch_paths": bp.value}

    def destroy(self) -> None:
        if self._h:
            N.call("cupbr_batch_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

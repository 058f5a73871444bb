"""Learned radiance cache: a small FP16 MLP trained online on the path
tracer's own radiance and queried to end paths early.

No counterpart in the reference; the renderer it shortens is
PBRendering::pathtracing (PathTracer.cu:97-169).  `RadianceCache` wraps
cupbr_cache_* of include/cupbr_c.h: tcgen05 inference and training kernels
(csrc/cache_mlp.cu), the cached shading stage (csrc/pathtracer.cu) and the
training-sample collection (csrc/cache.cu).

Record layout (5 float4 = 20 float32 per vertex, device memory):
  [0] position, -   [1] direction to the previous vertex, roughness
  [2] normal, bounces left (max trace depth - vertex depth)
  [3] diffuse albedo, -
  [4] training samples: target RGB, weight (0 or 1); inference: -
Parameters: layer-major, each layer row-major [out][in], see `LAYERS`.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _native as N

# (out, in) of each weight matrix as exposed through get/set_params
LAYERS = [(64, 96), (64, 64), (64, 64), (64, 64), (64, 64), (3, 64)]
RECORD_FLOATS = 20


def _ptr(v) -> Optional[C.c_void_p]:
    return C.c_void_p(v) if v else None


class RadianceCache:
    """cupbr_cache_t bound to a committed scene (its box scales the position
    encoding).  Defaults: 2^16 training samples per frame in Adam steps of
    2^14, learning rate 1e-2."""

    def __init__(self, scene, cache_depth: int = 1, train_stride: int = 32, batch: int = 1 << 14,
                 samples_per_frame: int = 1 << 16, learning_rate: float = 1e-2, seed: int = 0,
                 loss: str = "relative", weight_average: float = 0.0, cache_specular: bool = False,
                 train_suffix: int = 0):
        kinds = {"relative": 0, "l2": 1}
        if loss not in kinds:
            raise ValueError(f"loss must be one of {sorted(kinds)}")
        self.desc = N.CacheDesc(int(cache_depth), int(train_stride), int(batch), int(samples_per_frame),
                                float(learning_rate), int(seed), kinds[loss], float(weight_average),
                                1 if cache_specular else 0, int(train_suffix))
        h = C.c_void_p()
        N.call("cupbr_cache_create", scene._h, C.byref(self.desc), C.byref(h))
        self._h = h

    def destroy(self) -> None:
        if self._h:
            N.call("cupbr_cache_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    @staticmethod
    def param_count() -> int:
        return int(N.lib.cupbr_cache_param_count())

    def bounds(self):
        lo = (C.c_float * 3)()
        inv = (C.c_float * 3)()
        N.call("cupbr_cache_get_bounds", self._h, lo, inv)
        return np.asarray(lo[:], np.float32), np.asarray(inv[:], np.float32)

    def params(self) -> np.ndarray:
        out = np.empty(self.param_count(), np.float32)
        N.call("cupbr_cache_get_params", self._h, out.ctypes.data_as(C.c_void_p))
        return out

    def set_params(self, p) -> None:
        p = np.ascontiguousarray(p, np.float32)
        if p.size != self.param_count():
            raise ValueError(f"expected {self.param_count()} parameters, got {p.size}")
        N.call("cupbr_cache_set_params", self._h, p.ctypes.data_as(C.c_void_p))

    def save(self, path: str) -> None:
        N.call("cupbr_cache_save", self._h, path.encode())

    def load(self, path: str) -> None:
        N.call("cupbr_cache_load", self._h, path.encode())

    def infer(self, records_ptr: int, n: int, out_ptr: int, stream: Optional[int] = None) -> None:
        """out[i] (float4) = network RGB of record i."""
        N.call("cupbr_cache_infer", self._h, _ptr(records_ptr), int(n), _ptr(out_ptr), _ptr(stream))

    def train_step(self, samples_ptr: int, n: int, stream: Optional[int] = None) -> None:
        N.call("cupbr_cache_train_step", self._h, _ptr(samples_ptr), int(n), _ptr(stream))

    def gradient(self) -> np.ndarray:
        out = np.empty(self.param_count(), np.float32)
        N.call("cupbr_cache_get_gradient", self._h, out.ctypes.data_as(C.c_void_p))
        return out

    def loss(self):
        """(relative L2 loss, weighted samples) of the last Adam step."""
        l, w = C.c_float(), C.c_float()
        N.call("cupbr_cache_get_loss", self._h, C.byref(l), C.byref(w))
        return float(l.value), float(w.value)

    def render(self, scene, camera, width: int, height: int, frame0: int, frames: int, max_depth: int,
               image_ptr: int, train: bool = True, stream: Optional[int] = None) -> None:
        N.call("cupbr_cache_render", self._h, scene._h, C.byref(camera._c), int(width), int(height), int(frame0),
               int(frames), int(max_depth), 1 if train else 0, _ptr(image_ptr), _ptr(stream))

    def counters(self):
        """(tensor-core waits that ran out of time, queries, training samples of the last frame)"""
        out = (C.c_uint32 * 3)()
        N.call("cupbr_cache_get_counters", self._h, out)
        return tuple(int(v) for v in out)

    def check(self, stream=None) -> None:
        """Raises CupbrError (CUPBR_ERR_TIMEOUT) if a tensor-core wait ran out
        since the last check, and clears that count; CUPBR_ERR_STATE once the
        cache is lost (cupbr_cache_check)."""
        N.call("cupbr_cache_check", self._h, stream)

    def set_wait_probe(self, ns: int) -> None:
        """Test hook: inference CTAs wait `ns` on a barrier nothing arrives on
        and give up (cupbr_cache_set_wait_probe); 0 turns it off."""
        N.call("cupbr_cache_set_wait_probe", self._h, int(ns))

    def set_batch_paths(self, paths: int) -> None:
        """Paths per wavefront (whole frames, at least one; default 2^25)."""
        N.call("cupbr_cache_set_batch_paths", self._h, int(paths))

    def set_tail_paths(self, paths: int) -> None:
        """Ray queues below `paths` rays (default 2^16) finish their paths in
        one per-path launch; 0 never."""
        N.call("cupbr_cache_set_tail_paths", self._h, int(paths))

    def set_profiling(self, enable: bool) -> None:
        N.call("cupbr_cache_set_profiling", self._h, 1 if enable else 0)

    STAGES = ("camera", "extend", "shade", "connect", "infer", "accumulate_collect", "train")

    def stage_times(self):
        """{stage: ms} summed over the profiled wavefronts since the last
        call (stages as in STAGES; extend / shade / connect over all depths)
        and the wavefront count."""
        ms = (C.c_float * 7)()
        n = C.c_uint32()
        N.call("cupbr_cache_get_stage_times", self._h, ms, C.byref(n))
        return dict(zip(self.STAGES, (float(v) for v in ms))), int(n.value)

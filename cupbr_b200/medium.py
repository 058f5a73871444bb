"""Heterogeneous (density-grid) medium: forward rendering and gradients.

No counterpart in the reference, whose VolumeRenderer.cu renders a
homogeneous medium only and differentiates nothing.  `Medium` wraps
cupbr_medium_* of include/cupbr_c.h; `render` is a torch.autograd.Function
over the density grid (and the scene parameters: medium albedo, diffuse
albedos, light radiances) whose backward is the CUDA path-replay adjoint.

Device buffers are passed as raw pointers: torch tensors (CUDA, float32,
contiguous) through .data_ptr(), or cupbr device allocations.
"""
from __future__ import annotations

import ctypes as C
from typing import Optional

import numpy as np

from . import _native as N


class Medium:
    """cupbr_medium_t.  grid_shape = (nz, ny, nx); box = (lo, hi) in world
    space; q = 0 selects analog delta tracking (forward only), 0 < q < 1
    weighted tracking with real-event probability q (differentiable)."""

    def __init__(self, grid_shape, box, majorant: float, albedo: float = 0.9, g: float = 0.0, q: float = 0.5):
        nz, ny, nx = (int(v) for v in grid_shape)
        lo, hi = box
        self.shape = (nz, ny, nx)
        self.desc = N.MediumDesc(nx, ny, nz, N.Vec3.of(lo), N.Vec3.of(hi), float(majorant), float(albedo), float(g),
                                 float(q))
        h = C.c_void_p()
        N.call("cupbr_medium_create", C.byref(self.desc), C.byref(h))
        self._h = h

    def destroy(self) -> None:
        if self._h:
            N.call("cupbr_medium_destroy", self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.destroy()
        except Exception:
            pass

    @staticmethod
    def param_count(scene) -> int:
        n = C.c_uint32()
        N.call("cupbr_medium_param_count", scene._h, C.byref(n))
        return int(n.value)

    def params(self, scene) -> np.ndarray:
        """Current values of the parameter vector the gradient refers to:
        [albedo, per object albedo_d (3), per object albedo_e (3), per light
        radiance or intensity (3)]."""
        info = scene.info()
        out = [self.desc.albedo]
        for i in range(info["objects"]):
            out += list(scene.object(i).material.albedo_d.tuple())
        for i in range(info["objects"]):
            out += list(scene.object(i).material.albedo_e.tuple())
        for i in range(info["lights"]):
            li = scene.light(i)
            out += list((li.intensity if li.type == 0 else li.radiance).tuple())
        return np.asarray(out, np.float32)

    def forward(self, scene, density_ptr: int, camera, width: int, height: int, spp: int, frame0: int,
                max_depth: int, image_ptr: int, stream: Optional[int] = None) -> None:
        N.call("cupbr_medium_forward", self._h, scene._h, C.c_void_p(density_ptr), C.byref(camera._c), width, height,
               spp, frame0, max_depth, C.c_void_p(image_ptr), C.c_void_p(stream) if stream else None)

    def backward(self, scene, density_ptr: int, camera, width: int, height: int, spp: int, frame0: int,
                 max_depth: int, grad_image_ptr: int, grad_density_ptr: int, grad_params_ptr: int,
                 stream: Optional[int] = None) -> None:
        N.call("cupbr_medium_backward", self._h, scene._h, C.c_void_p(density_ptr), C.byref(camera._c), width,
               height, spp, frame0, max_depth, C.c_void_p(grad_image_ptr), C.c_void_p(grad_density_ptr),
               C.c_void_p(grad_params_ptr), C.c_void_p(stream) if stream else None)

    def set_batch_paths(self, paths: int) -> None:
        N.call("cupbr_medium_set_batch_paths", self._h, int(paths))

    def set_profiling(self, enable: bool) -> None:
        N.call("cupbr_medium_set_profiling", self._h, int(bool(enable)))

    def stage_times(self) -> dict:
        """Summed stage times (ms) of the forward calls made while profiling."""
        ms = (C.c_float * 6)()
        wf, launches = C.c_uint32(), C.c_uint32()
        N.call("cupbr_medium_get_stage_times", self._h, ms, C.byref(wf), C.byref(launches))
        out = dict(zip(("camera", "extend", "shade", "transmit", "connect", "accumulate"), list(ms)))
        out["wavefronts"], out["shade_launches"] = wf.value, launches.value
        return out

    def set_instrumented(self, enable: bool) -> None:
        N.call("cupbr_medium_set_instrumented", self._h, int(bool(enable)))

    def stats(self) -> dict:
        """Counts of the forward calls made while instrumented (then cleared)."""
        v = (C.c_uint64 * 5)()
        N.call("cupbr_medium_get_stats", self._h, v)
        return dict(zip(("flight_lookups", "ratio_lookups", "vertices", "shadow_rays", "paths"), list(v)))

    def error_count(self) -> int:
        n = C.c_uint32()
        N.call("cupbr_medium_get_error_count", self._h, C.byref(n))
        return int(n.value)


def _function():
    import torch

    class _Render(torch.autograd.Function):
        @staticmethod
        def forward(ctx, density, params, medium, scene, camera, width, height, spp, frame0, max_depth):
            if not density.is_cuda or density.dtype != torch.float32 or tuple(density.shape) != medium.shape:
                raise ValueError(f"density must be a CUDA float32 tensor of shape {medium.shape}")
            density = density.contiguous()
            img = torch.empty((height, width, 3), device=density.device, dtype=torch.float32)
            stream = torch.cuda.current_stream(density.device).cuda_stream
            medium.forward(scene, density.data_ptr(), camera, width, height, spp, frame0, max_depth,
                           img.data_ptr(), stream)
            ctx.save_for_backward(density)
            ctx.args = (medium, scene, camera, width, height, spp, frame0, max_depth, params.shape)
            return img

        @staticmethod
        def backward(ctx, grad_img):
            (density,) = ctx.saved_tensors
            medium, scene, camera, width, height, spp, frame0, max_depth, pshape = ctx.args
            gi = grad_img.contiguous().to(torch.float32)
            gd = torch.zeros_like(density)
            gp = torch.zeros(pshape, device=density.device, dtype=torch.float32)
            stream = torch.cuda.current_stream(density.device).cuda_stream
            medium.backward(scene, density.data_ptr(), camera, width, height, spp, frame0, max_depth, gi.data_ptr(),
                            gd.data_ptr(), gp.data_ptr(), stream)
            return gd, gp, None, None, None, None, None, None, None, None

    return _Render


_RENDER = None


def render(density, params, medium: Medium, scene, camera, width: int, height: int, spp: int = 1, frame0: int = 0,
           max_depth: int = 5):
    """Differentiable grid-medium render: (height, width, 3) float32 image.

    `params` is a CUDA tensor holding Medium.params(scene); the forward pass
    reads the values stored in the scene and medium (params only carries the
    gradient), so rebuild the scene / medium after changing them."""
    global _RENDER
    if _RENDER is None:
        _RENDER = _function()
    return _RENDER.apply(density, params, medium, scene, camera, width, height, spp, frame0, max_depth)

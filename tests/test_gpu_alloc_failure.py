"""Allocation failures made on the host (cupbr_debug_fail_allocation): every
device allocation of the library goes through one allocator, which the test
makes fail at the n-th allocation from now, for n = 0, 1, 2, ... until a
scenario (scene commit with the GPU BVH build, renderer set-up, a
pipelined two-frame render, tone map) gets through without meeting it.
Every failing run must raise CupbrError with CUPBR_ERR_CUDA and an
out-of-memory message, the run that gets through must give the image of an
undisturbed run bit for bit, and afterwards the device's free memory must
be back where it was (within 8 MB: the smallest buffers of the scenario
are below the driver's reporting granularity, its workspaces are not).
No GPU fault is involved: the allocator returns the error instead of
calling cudaMalloc."""
import gc

import numpy as np
import pytest

import cupbr_b200 as cb
from cupbr_b200 import _native as N
from cupbr_b200 import scenes

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")


def scenario():
    sc = scenes.cornell_box().build()
    r = cb.PBRenderer(cb.RenderingMethod.PATHTRACER)
    try:
        r.set_output_size(320, 256)
        r.register_scene(sc)
        r.set_method(cb.RenderingMethod.PATHTRACER)
        r.set_max_trace_depth(5)
        r.set_russian_roulette(False)
        r.set_pipelined(True)
        r.render_frames(cb.Camera(320, 256), 2)
        tm = cb.ToneMapper(cb.ToneMappingType.REINHARD)
        tm.register_image(r.get_output_image())
        tm.tone_map()
        return r.get_output_image().numpy(), tm.get_render_buffer().numpy()
    finally:
        del r
        sc.destroy()


def test_injected_allocation_failures_are_reported_and_leak_nothing():
    ref = scenario()
    gc.collect()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    failures = 0
    try:
        for n in range(400):
            N.call("cupbr_debug_fail_allocation", n)
            try:
                got = scenario()
            except cb.CupbrError as e:
                assert e.code == -2, str(e)                      # CUPBR_ERR_CUDA
                assert "memory" in str(e).lower(), str(e)
                failures += 1
                gc.collect()
                continue
            # this run did not reach the n-th allocation: the scenario makes n
            assert np.array_equal(got[0], ref[0]) and np.array_equal(got[1], ref[1])
            break
        else:
            pytest.fail("the scenario never got through")
    finally:
        N.call("cupbr_debug_fail_allocation", -1)
    print(f"{failures} injected allocation failures, each reported")
    assert failures >= 10
    gc.collect()
    torch.cuda.synchronize()
    free1 = torch.cuda.mem_get_info()[0]
    assert abs(free1 - free0) <= 8 << 20, (free0, free1)

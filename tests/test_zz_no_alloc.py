"""cupbr_bloom_noalloc: bloom for callers that cannot allocate device memory
(applications that hand out a pre-reserved device budget themselves, frame
loops that must not allocate after start-up).  Its scratch is a fixed array
inside the library, so the call itself allocates nothing; the test allocates
only the caller-owned input and output buffers.

Checked through the C ABI against the allocating entry point
(cupbr_postprocessor_bloom) on two calls in a row -- a large image, then a
smaller odd-sized one, so leftovers of the first call in the shared scratch
would show -- with the bar the bloom tests use: bit-exact.  This file is
collected last so that a run stopping at the first failure has run every
other test already.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _dev(nbytes):
    from cupbr_b200 import _native as N
    p = C.c_void_p()
    N.call("cupbr_device_alloc", C.byref(p), nbytes)
    return p


def test_bloom_noalloc_matches_allocating_bloom_twice():
    import cupbr_b200 as cb
    from cupbr_b200 import _native as N

    th = (C.c_float * 4)(*[float(x) for x in cb.threshold_curve(0.9, 0.6)])
    for w, h, seed in ((1920, 1080, 1), (641, 359, 2)):
        rng = np.random.default_rng(seed)
        hdr = np.ascontiguousarray((rng.random((h, w, 3), dtype=np.float32) * 2.2) ** 3)
        src = _dev(hdr.nbytes)
        out = _dev(hdr.nbytes)
        try:
            N.call("cupbr_memcpy_h2d", src, hdr.ctypes.data, hdr.nbytes, None)
            N.call("cupbr_stream_synchronize", None)
            pp = cb.PostProcessor()
            pp.register_image(cb.DeviceImage(src.value, w, h, 3, np.float32))
            pp.bloom(cb.threshold_curve(0.9, 0.6))
            ref = pp.get_post_process_buffer().numpy()
            N.call("cupbr_bloom_noalloc", src, w, h, th, out, None)
            got = np.empty_like(hdr)
            N.call("cupbr_memcpy_d2h", got.ctypes.data, out, got.nbytes, None)
            N.call("cupbr_stream_synchronize", None)
            assert np.array_equal(got, ref), f"{w}x{h}: max diff {np.abs(got - ref).max()}"
            del pp
        finally:
            N.call("cupbr_device_free", src)
            N.call("cupbr_device_free", out)


def test_bloom_noalloc_rejects_oversized_images():
    import cupbr_b200 as cb
    from cupbr_b200 import _native as N

    th = (C.c_float * 4)(1.0, 0.0, 2.0, 0.25)
    with pytest.raises(cb.CupbrError, match="too large"):
        N.call("cupbr_bloom_noalloc", C.c_void_p(16), 4096, 2050, th, C.c_void_p(16), None)

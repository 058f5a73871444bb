// Bloom and tone mapping (PostProcessor::bloom, ToneMapper::toneMap).
//
// The reference builds a 6-level pyramid with 12 launches and 2 device
// copies (PostProcessor.cpp:125-142, PyramidConstructor.cu:9-169), but its
// upscale step reads pyramid_down[d + 1] (PyramidConstructor.cu:84), so the
// output only depends on levels 0 and 1:
//     out = hdr + T(hdr) + tent3x3(box2x2(T(hdr))) / 16
// with T the soft-knee threshold.  Here that is two passes: k_bloom_down
// builds the half-resolution level-1 image straight from the HDR input
// (thresholding its four taps on the fly), and k_bloom_up forms the output,
// optionally tone-mapping it in the same pass.  The float operations and
// their order are the reference's, so results match it exactly.
#include "post.hpp"

#include <mutex>

#include "dev_common.cuh"

namespace cupbr_b200 {

namespace {

// thresholding_kernel, PyramidConstructor.cu:9-30
__device__ __forceinline__ f3 threshold(f3 c, float4 th) {
    float br = c.x > c.y ? c.x : c.y;
    br = c.z > br ? c.z : br;
    float rq = clampf(br - th.y, 0.0f, th.z);
    rq = th.w * rq * rq;
    float s = fmaxf(rq, br - th.x) / fmaxf(br, 1e-5f);
    return mk(c.x * s, c.y * s, c.z * s);
}

__device__ __forceinline__ f3 ld3(const float* p) { return mk(p[0], p[1], p[2]); }

// ToneMapper.cu:17-41 (REINHARD) and :43-69 (GAMMA)
__device__ __forceinline__ uchar4 tonemap_px(f3 c, int type, float exposure) {
    float v[3] = {c.x, c.y, c.z};
    uint8_t o[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        float m;
        if (type == 0) {
            const float e = (k == 2) ? (float)(1.0f / 2.2) : 1.0f / 2.2f;
            m = powf((float)(1.0 - (double)expf(-v[k] * exposure)), e);
        } else {
            const float x = v[k];
            m = x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.0f / 2.4f) - 0.055f;
        }
        o[k] = (uint8_t)(clampf(m, 0.0f, 1.0f) * 255.0f);
    }
    return make_uchar4(o[0], o[1], o[2], 255);
}

__global__ void k_tonemap(const float* __restrict__ hdr, uint32_t n, int type, float exposure, uchar4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = tonemap_px(ld3(hdr + 3 * (size_t)i), type, exposure);
}

// downsample_kernel (PyramidConstructor.cu:32-65) of the thresholded level 0
__global__ void k_bloom_down(const float* __restrict__ hdr, uint32_t w, uint32_t h, float4 th, float* __restrict__ d1,
                             uint32_t w2, uint32_t h2) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w2 * h2) return;
    const uint32_t y = i / w2, x = i - w2 * y;
    f3 r = splat(0.0f);
    const uint32_t ox[4] = {0, 0, 1, 1}, oy[4] = {0, 1, 0, 1};
#pragma unroll
    for (int k = 0; k < 4; ++k) {
        uint32_t sx = 2 * x + ox[k], sy = 2 * y + oy[k];
        if (sx >= w) sx = w - 1;
        if (sy >= h) sy = h - 1;
        r += threshold(ld3(hdr + 3 * ((size_t)sx + (size_t)sy * w)), th);
    }
    float* o = d1 + 3 * (size_t)i;
    o[0] = r.x / 4.0f; o[1] = r.y / 4.0f; o[2] = r.z / 4.0f;
}

// upscale_and_combine_kernel at level 0 (PyramidConstructor.cu:67-112)
// followed by combine_kernel (:114-125); TONEMAP fuses ToneMapper::toneMap.
template <bool TONEMAP>
__global__ void k_bloom_up(const float* __restrict__ hdr, uint32_t w, uint32_t h, float4 th, const float* __restrict__ d1,
                           uint32_t w2, uint32_t h2, float* __restrict__ out, uchar4* __restrict__ out8, int type,
                           float exposure) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= w * h) return;
    const int32_t y = (int32_t)(i / w), x = (int32_t)(i - w * (uint32_t)y);
    const int32_t dx = x / 2, dy = y / 2;
    const float kern[3][3] = {{1.0f, 2.0f, 1.0f}, {2.0f, 4.0f, 2.0f}, {1.0f, 2.0f, 1.0f}};
    f3 r = splat(0.0f);
#pragma unroll
    for (int32_t u = -1; u < 2; ++u)
#pragma unroll
        for (int32_t v = -1; v < 2; ++v) {
            int32_t sx = dx + u, sy = dy + v;
            if (sx < 0) sx = 0;
            if (sx >= (int32_t)w2) sx = (int32_t)w2 - 1;
            if (sy < 0) sy = 0;
            if (sy >= (int32_t)h2) sy = (int32_t)h2 - 1;
            r += ld3(d1 + 3 * ((size_t)sx + (size_t)sy * w2)) * kern[u + 1][v + 1];
        }
    const f3 c = ld3(hdr + 3 * (size_t)i);
    const f3 up = r / 16.0f + threshold(c, th);
    const f3 res = c + up;
    if (TONEMAP) {
        out8[i] = tonemap_px(res, type, exposure);
    } else {
        float* o = out + 3 * (size_t)i;
        o[0] = res.x; o[1] = res.y; o[2] = res.z;
    }
}

// Level-1 scratch for the bloom entry point that allocates nothing
// (bloom_static_scratch below).  It lives in the module's global memory:
// every GPU that loads the library holds these 12 MiB until the process
// exits.  Host code must not pass this symbol to a kernel directly: on the
// host it names a host-side stand-in, not the device address.
static __device__ __align__(256) float g_bloom_scratch[3 * BLOOM_NOALLOC_MAX_HALF_PIXELS];

std::mutex g_scratch_mutex;
float* g_scratch_ptr[BLOOM_NOALLOC_MAX_DEVICES] = {};

}  // namespace

cudaError_t bloom_static_scratch(const float* hdr, uint32_t w, uint32_t h, const float th[4], float* out,
                                 cudaStream_t st) {
    // Set-up, once per device: ask the runtime for the device address of
    // the scratch array with the caller's device current.
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= BLOOM_NOALLOC_MAX_DEVICES) return cudaErrorInvalidDevice;
    float* scratch = nullptr;
    {
        std::lock_guard<std::mutex> lock(g_scratch_mutex);
        if (!g_scratch_ptr[dev]) {
            void* p = nullptr;
            e = cudaGetSymbolAddress(&p, g_bloom_scratch);
            if (e != cudaSuccess) return e;
            g_scratch_ptr[dev] = static_cast<float*>(p);
        }
        scratch = g_scratch_ptr[dev];
    }
    // k_bloom_down writes every scratch element that k_bloom_up reads, so
    // nothing left over from an earlier call needs clearing.
    const uint32_t w2 = w / 2, h2 = h / 2;
    const float4 t4 = make_float4(th[0], th[1], th[2], th[3]);
    k_bloom_down<<<(w2 * h2 + 255) / 256, 256, 0, st>>>(hdr, w, h, t4, scratch, w2, h2);
    k_bloom_up<false><<<(w * h + 255) / 256, 256, 0, st>>>(hdr, w, h, t4, scratch, w2, h2, out, nullptr, 0, 0.0f);
    return cudaGetLastError();
}

cudaError_t launch_tonemap(const float* hdr, uint32_t npix, int type, float exposure, uint8_t* rgba, cudaStream_t st) {
    if (npix == 0) return cudaSuccess;
    k_tonemap<<<(npix + 255) / 256, 256, 0, st>>>(hdr, npix, type, exposure, reinterpret_cast<uchar4*>(rgba));
    return cudaGetLastError();
}

cudaError_t launch_bloom(const float* hdr, uint32_t w, uint32_t h, const float th[4], float* scratch_half, float* out,
                         uint8_t* rgba, int type, float exposure, cudaStream_t st) {
    const uint32_t w2 = w / 2, h2 = h / 2;
    const float4 t4 = make_float4(th[0], th[1], th[2], th[3]);
    const uint32_t n2 = w2 * h2, n = w * h;
    k_bloom_down<<<(n2 + 255) / 256, 256, 0, st>>>(hdr, w, h, t4, scratch_half, w2, h2);
    if (rgba)
        k_bloom_up<true><<<(n + 255) / 256, 256, 0, st>>>(hdr, w, h, t4, scratch_half, w2, h2, nullptr,
                                                         reinterpret_cast<uchar4*>(rgba), type, exposure);
    else
        k_bloom_up<false><<<(n + 255) / 256, 256, 0, st>>>(hdr, w, h, t4, scratch_half, w2, h2, out, nullptr, 0, 0.0f);
    return cudaGetLastError();
}

}  // namespace cupbr_b200

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

// ToneMapper.cu:17-41 (REINHARD) and :43-69 (GAMMA), channel k of one pixel
__device__ __forceinline__ uint8_t tone_direct(float x, int type, float exposure, int k) {
    float m;
    if (type == 0) {
        const float e = (k == 2) ? (float)(1.0f / 2.2) : 1.0f / 2.2f;
        m = powf((float)(1.0 - (double)expf(-x * exposure)), e);
    } else {
        m = x <= 0.0031308f ? 12.92f * x : 1.055f * powf(x, 1.0f / 2.4f) - 0.055f;
    }
    return (uint8_t)(clampf(m, 0.0f, 1.0f) * 255.0f);
}

// ---- tone-map levels from tables
//
// A channel's 8-bit level is a step function of u = x * exposure (REINHARD:
// tone_direct evaluates expf(-x * exposure), and (-x) * e == -(x * e)) or of
// u = x (GAMMA).  For u in [2^-20, 2^5) a table holds one 32-bit word per
// bucket of 2^16 consecutive float bit patterns (128 buckets per octave):
// the level at the bucket's first float (bits 17-24) and the offset of the
// one level step inside the bucket (bits 0-16; 2^16 when there is none).
// k_tone_levels_build makes the tables by evaluating tone_direct at every
// float of that range on the device, so a looked-up level is tone_direct's
// level.  Below 2^-20 every formula gives level 0 (REINHARD:
// (2^-20)^(1/2.2) * 255 < 0.5; GAMMA: 12.92 * 2^-20 * 255 < 0.01), from 2^5
// up (+inf included) level 255 (REINHARD: 1 - e^-32 rounds to 1; GAMMA: the
// power term exceeds 4); negative inputs, NaN and the buckets the build
// flags (bit 25: a decrease or more than one step inside) take the
// formulas.  cupbr_tonemap_verify_levels compares both for every 32-bit
// input.  Tables: 0 REINHARD red / green, 1 REINHARD blue (its exponent
// rounds differently), 2 GAMMA; 12.8 KB each, so the bloom output kernel
// keeps the ones it needs in shared memory, where lanes with unrelated
// values cost a few bank conflicts instead of one L1 line each.
constexpr uint32_t TONE_LO_BITS = 0x35800000u;  // 2^-20
constexpr uint32_t TONE_HI_BITS = 0x42000000u;  // 2^5
constexpr uint32_t TONE_INF_BITS = 0x7f800000u;
constexpr uint32_t TONE_SHIFT = 16;
constexpr uint32_t TONE_BUCKETS = (TONE_HI_BITS - TONE_LO_BITS) >> TONE_SHIFT;  // 3200
constexpr uint32_t TONE_NO_STEP = 1u << TONE_SHIFT;
constexpr uint32_t TONE_FLAG = 1u << 25;  // this bucket takes the formulas
constexpr int TONE_TABLES = 3;
static __device__ __align__(16) uint32_t g_tone_levels[TONE_TABLES][TONE_BUCKETS];
// 1 once g_tone_levels is complete; until then (and after a device reset
// reloads the module) the kernels use the formulas.
static __device__ uint32_t g_tone_ready;

__device__ __forceinline__ bool tone_tables_ready() {
    uint32_t v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(&g_tone_ready) : "memory");
    return v != 0;
}

// The two tables a tone-map type reads: REINHARD red / green and blue, or
// GAMMA for every channel.
struct ToneTables {
    const uint32_t* rg;
    const uint32_t* b;
};
__device__ __forceinline__ ToneTables tone_tables_global(int type) {
    return type == 0 ? ToneTables{g_tone_levels[0], g_tone_levels[1]} : ToneTables{g_tone_levels[2], g_tone_levels[2]};
}
// Bytes of shared memory stage_tone_tables fills for a type.
__host__ __device__ constexpr uint32_t tone_smem_bytes(int type) {
    return (type == 0 ? 2u : 1u) * TONE_BUCKETS * (uint32_t)sizeof(uint32_t);
}
// Copies the type's tables into s (tone_smem_bytes(type) bytes) when the
// tables are complete; block-uniform, with __syncthreads inside.  Returns
// false (tables not yet built) to every thread of the block otherwise.
__device__ __forceinline__ bool stage_tone_tables(uint32_t* s, int type, ToneTables& tt) {
    __shared__ uint32_t s_ready;
    if (threadIdx.x == 0) s_ready = tone_tables_ready() ? 1u : 0u;
    __syncthreads();
    if (!s_ready) return false;
    const uint4* src = reinterpret_cast<const uint4*>(type == 0 ? g_tone_levels[0] : g_tone_levels[2]);
    uint4* dst = reinterpret_cast<uint4*>(s);
    const uint32_t n16 = tone_smem_bytes(type) / 16;  // the two REINHARD tables are adjacent
    for (uint32_t i = threadIdx.x; i < n16; i += blockDim.x) dst[i] = src[i];
    __syncthreads();
    tt = type == 0 ? ToneTables{s, s + TONE_BUCKETS} : ToneTables{s, s};
    return true;
}

__device__ __forceinline__ uint8_t tone_lookup(float x, int type, float exposure, int k, const uint32_t* tbl) {
    const float u = type == 0 ? x * exposure : x;
    const uint32_t b = __float_as_uint(u);
    if (b < TONE_LO_BITS) return 0;
    if (b < TONE_HI_BITS) {
        const uint32_t e = tbl[(b - TONE_LO_BITS) >> TONE_SHIFT];
        if (!(e & TONE_FLAG))
            return (uint8_t)(((e >> 17) & 0xffu) + ((b & (TONE_NO_STEP - 1)) >= (e & 0x1ffffu) ? 1u : 0u));
    } else if (b <= TONE_INF_BITS) {
        return 255;
    }
    return tone_direct(x, type, exposure, k);
}

__device__ __forceinline__ uchar4 tonemap_px(f3 c, int type, float exposure, bool tables, const ToneTables& tt) {
    if (tables)
        return make_uchar4(tone_lookup(c.x, type, exposure, 0, tt.rg), tone_lookup(c.y, type, exposure, 1, tt.rg),
                           tone_lookup(c.z, type, exposure, 2, tt.b), 255);
    return make_uchar4(tone_direct(c.x, type, exposure, 0), tone_direct(c.y, type, exposure, 1),
                       tone_direct(c.z, type, exposure, 2), 255);
}

// One block per (bucket, table): 256 threads evaluate tone_direct at 256
// consecutive floats each and report the bucket's steps.
__global__ void __launch_bounds__(256) k_tone_levels_build() {
    const uint32_t q = blockIdx.x, t = blockIdx.y;
    const uint32_t first = TONE_LO_BITS + (q << TONE_SHIFT);
    constexpr uint32_t per = (1u << TONE_SHIFT) / 256;
    const uint32_t b0 = first + threadIdx.x * per;
    const int type = t == 2 ? 1 : 0, k = t == 1 ? 2 : 0;
    uint32_t prev = tone_direct(__uint_as_float(threadIdx.x == 0 ? b0 : b0 - 1), type, 1.0f, k);
    uint32_t steps = 0, bad = 0, pos = TONE_INF_BITS;
    for (uint32_t i = 0; i < per; ++i) {
        const uint32_t cur = tone_direct(__uint_as_float(b0 + i), type, 1.0f, k);
        if (cur < prev) bad = 1;
        if (cur > prev) {
            steps += cur - prev;
            if (pos == TONE_INF_BITS) pos = b0 + i;
        }
        prev = cur;
    }
    __shared__ uint32_t s_steps, s_bad, s_pos;
    if (threadIdx.x == 0) {
        s_steps = 0;
        s_bad = 0;
        s_pos = TONE_INF_BITS;
    }
    __syncthreads();
    if (steps) {
        atomicAdd(&s_steps, steps);
        atomicMin(&s_pos, pos);
    }
    if (bad) atomicOr(&s_bad, 1u);
    __syncthreads();
    if (threadIdx.x == 0) {
        const uint32_t base = tone_direct(__uint_as_float(first), type, 1.0f, k);
        const bool ok = s_bad == 0 && s_steps <= 1;
        const uint32_t off = s_steps ? s_pos - first : TONE_NO_STEP;  // 1 .. 2^16
        g_tone_levels[t][q] = ok ? (base << 17) | off : TONE_FLAG;
    }
}

__global__ void k_tone_levels_publish() {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(&g_tone_ready), "r"(1u) : "memory");
}

// Every 32-bit input of every table: the looked-up level against the
// formula's (inputs spread over the grid's threads, counts per table).
__global__ void k_tone_levels_verify(unsigned long long* __restrict__ mismatches) {
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned long long miss[TONE_TABLES] = {0, 0, 0};
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (1ull << 32); i += stride) {
        const float x = __uint_as_float((uint32_t)i);
#pragma unroll
        for (int t = 0; t < TONE_TABLES; ++t) {
            const int type = t == 2 ? 1 : 0, k = t == 1 ? 2 : 0;
            miss[t] += tone_lookup(x, type, 1.0f, k, g_tone_levels[t]) != tone_direct(x, type, 1.0f, k);
        }
    }
#pragma unroll
    for (int t = 0; t < TONE_TABLES; ++t)
        if (miss[t]) atomicAdd(&mismatches[t], miss[t]);
}

__global__ void k_tonemap(const float* __restrict__ hdr, uint32_t n, int type, float exposure, uchar4* __restrict__ out) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    out[i] = tonemap_px(ld3(hdr + 3 * (size_t)i), type, exposure, tone_tables_ready(), tone_tables_global(type));
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
        out8[i] = tonemap_px(res, type, exposure, tone_tables_ready(), tone_tables_global(type));
    } else {
        float* o = out + 3 * (size_t)i;
        o[0] = res.x; o[1] = res.y; o[2] = res.z;
    }
}

// ---- vectorised variants (image width a multiple of 4): the same float
// operations in the same order per pixel, with 128-bit loads and stores of
// four pixels (48 bytes of RGB) per thread.

__device__ __forceinline__ void ld12(const float* __restrict__ p, f3 v[4]) {
    const float4* q = reinterpret_cast<const float4*>(p);
    const float4 a = __ldg(q), b = __ldg(q + 1), c = __ldg(q + 2);
    v[0] = mk(a.x, a.y, a.z);
    v[1] = mk(a.w, b.x, b.y);
    v[2] = mk(b.z, b.w, c.x);
    v[3] = mk(c.y, c.z, c.w);
}
__device__ __forceinline__ void st12(float* __restrict__ p, const f3 v[4]) {
    float4* q = reinterpret_cast<float4*>(p);
    q[0] = make_float4(v[0].x, v[0].y, v[0].z, v[1].x);
    q[1] = make_float4(v[1].y, v[1].z, v[2].x, v[2].y);
    q[2] = make_float4(v[2].z, v[3].x, v[3].y, v[3].z);
}

// One quad of pixels per thread, the level tables read through L1: rendered
// images are smooth, so a warp's lookups share few table lines, and the
// kernel leaves the L1 of the SMs it shares with a renderer's traversal
// kernels (pipelined render()) as it is.
__global__ void k_tonemap4(const float* __restrict__ hdr, uint32_t n, int type, float exposure,
                           uchar4* __restrict__ out) {
    const uint32_t i4 = blockIdx.x * blockDim.x + threadIdx.x;  // pixels 4 i4 .. 4 i4 + 3
    const bool tables = tone_tables_ready();
    const ToneTables tt = tone_tables_global(type);
    if (4 * i4 + 3 < n) {
        f3 v[4];
        ld12(hdr + 12 * (size_t)i4, v);
        uchar4 o[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) o[k] = tonemap_px(v[k], type, exposure, tables, tt);
        reinterpret_cast<uint4*>(out)[i4] = make_uint4(*reinterpret_cast<uint32_t*>(&o[0]),
                                                       *reinterpret_cast<uint32_t*>(&o[1]),
                                                       *reinterpret_cast<uint32_t*>(&o[2]),
                                                       *reinterpret_cast<uint32_t*>(&o[3]));
    } else {
        for (uint32_t i = 4 * i4; i < n; ++i) out[i] = tonemap_px(ld3(hdr + 3 * (size_t)i), type, exposure, tables, tt);
    }
}

// k_bloom_down for two neighbouring level-1 pixels (2 j, 2 j + 1) of row y:
// full-resolution columns 4 j .. 4 j + 3 of rows 2 y and 2 y + 1 (w % 4 ==
// 0, so no tap needs the edge clamp).
__global__ void k_bloom_down4(const float* __restrict__ hdr, uint32_t w, uint32_t h, float4 th,
                              float* __restrict__ d1, uint32_t w2, uint32_t h2) {
    const uint32_t pairs = w2 / 2;
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= pairs * h2) return;
    const uint32_t y = i / pairs, j = i - pairs * y;
    f3 a[4], b[4];
    ld12(hdr + 3 * ((size_t)(2 * y) * w + 4 * j), a);
    ld12(hdr + 3 * ((size_t)(2 * y + 1) * w + 4 * j), b);
    f3 r[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        // taps in the order (2x, 2y), (2x, 2y + 1), (2x + 1, 2y), (2x + 1, 2y + 1)
        f3 t = splat(0.0f);
        t += threshold(a[2 * k], th);
        t += threshold(b[2 * k], th);
        t += threshold(a[2 * k + 1], th);
        t += threshold(b[2 * k + 1], th);
        r[k] = mk(t.x / 4.0f, t.y / 4.0f, t.z / 4.0f);
    }
    float2* o = reinterpret_cast<float2*>(d1 + 3 * ((size_t)y * w2 + 2 * j));
    o[0] = make_float2(r[0].x, r[0].y);
    o[1] = make_float2(r[0].z, r[1].x);
    o[2] = make_float2(r[1].y, r[1].z);
}

// k_bloom_up for four pixels 4 j .. 4 j + 3 of row y: their level-1
// centres are columns 2 j and 2 j + 1, so one 4 x 3 neighbourhood of
// level-1 texels serves all four tent filters.
// k_bloom_up for the quads 4 j .. 4 j + 3 of the two rows 2 yp and 2 yp + 1:
// all eight pixels take their tent filter from level-1 row yp, and the
// quad's level-1 centres are columns 2 j and 2 j + 1, so one 4 x 3
// neighbourhood of level-1 texels and two filtered values serve them all.
// With TONEMAP, grid-stride with the level tables staged in shared memory as
// in shared memory (stage_tone_tables); without, one quad pair per thread.
template <bool TONEMAP>
__global__ void k_bloom_up4(const float* __restrict__ hdr, uint32_t w, uint32_t h, float4 th,
                            const float* __restrict__ d1, uint32_t w2, uint32_t h2, float* __restrict__ out,
                            uchar4* __restrict__ out8, int type, float exposure) {
    extern __shared__ __align__(16) uint32_t s_tone[];
    ToneTables tt{};
    bool tables = false;
    if (TONEMAP) tables = stage_tone_tables(s_tone, type, tt);
    const uint32_t quads = w / 4, row_pairs = (h + 1) / 2;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < quads * row_pairs; i += gridDim.x * blockDim.x) {
        const int32_t yp = (int32_t)(i / quads), j = (int32_t)(i - quads * (uint32_t)yp);
        const int32_t dy = yp;  // (2 yp) / 2 == (2 yp + 1) / 2
        const float kern[3][3] = {{1.0f, 2.0f, 1.0f}, {2.0f, 4.0f, 2.0f}, {1.0f, 2.0f, 1.0f}};
        f3 nb[4][3];  // level-1 columns 2j-1 .. 2j+2 (clamped) x rows dy-1 .. dy+1 (clamped)
#pragma unroll
        for (int cx = 0; cx < 4; ++cx)
#pragma unroll
            for (int cy = 0; cy < 3; ++cy) {
                int32_t sx = 2 * j - 1 + cx, sy = dy - 1 + cy;
                if (sx < 0) sx = 0;
                if (sx >= (int32_t)w2) sx = (int32_t)w2 - 1;
                if (sy < 0) sy = 0;
                if (sy >= (int32_t)h2) sy = (int32_t)h2 - 1;
                nb[cx][cy] = ld3(d1 + 3 * ((size_t)sx + (size_t)sy * w2));
            }
        f3 rr[2];  // tent-filtered level 1 at columns 2 j and 2 j + 1
#pragma unroll
        for (int base = 0; base < 2; ++base) {
            f3 r = splat(0.0f);
            // r += nb * kern, the product exact (a weight of 1, 2 or 4), so one
            // fused multiply-add rounds exactly as the reference's multiply then add
#pragma unroll
            for (int u = 0; u < 3; ++u)
#pragma unroll
                for (int v = 0; v < 3; ++v) {
                    const f3 a = nb[base + u][v];
                    const float kw = kern[u][v];
                    r = mk(__fmaf_rn(a.x, kw, r.x), __fmaf_rn(a.y, kw, r.y), __fmaf_rn(a.z, kw, r.z));
                }
            rr[base] = r;
        }
#pragma unroll
        for (int yy = 0; yy < 2; ++yy) {
            const int32_t y = 2 * yp + yy;
            if (y >= (int32_t)h) break;
            f3 c[4];
            ld12(hdr + 3 * ((size_t)y * w + 4 * j), c);
            f3 res[4];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                const f3 up = rr[k / 2] / 16.0f + threshold(c[k], th);
                res[k] = c[k] + up;
            }
            const size_t p0 = (size_t)y * w + 4 * (size_t)j;
            if (TONEMAP) {
                uchar4 o[4];
#pragma unroll
                for (int k = 0; k < 4; ++k) o[k] = tonemap_px(res[k], type, exposure, tables, tt);
                *reinterpret_cast<uint4*>(out8 + p0) = make_uint4(*reinterpret_cast<uint32_t*>(&o[0]),
                                                                   *reinterpret_cast<uint32_t*>(&o[1]),
                                                                   *reinterpret_cast<uint32_t*>(&o[2]),
                                                                   *reinterpret_cast<uint32_t*>(&o[3]));
            } else {
                st12(out + 3 * p0, res);
            }
        }
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

std::mutex g_tone_mutex;
bool g_tone_enqueued[BLOOM_NOALLOC_MAX_DEVICES] = {};

}  // namespace

cudaError_t ensure_tone_levels(cudaStream_t st) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= BLOOM_NOALLOC_MAX_DEVICES) return cudaSuccess;  // the kernels use the formulas
    std::lock_guard<std::mutex> lock(g_tone_mutex);
    if (g_tone_enqueued[dev]) return cudaSuccess;
    // ~0.6 G formula evaluations, once per device (about a millisecond);
    // kernels on other streams use the formulas until the publish runs.
    k_tone_levels_build<<<dim3(TONE_BUCKETS, TONE_TABLES), 256, 0, st>>>();
    k_tone_levels_publish<<<1, 1, 0, st>>>();
    e = cudaGetLastError();
    if (e == cudaSuccess) g_tone_enqueued[dev] = true;
    return e;
}

cudaError_t verify_tone_levels(unsigned long long mismatches[3], uint32_t flagged[3], cudaStream_t st) {
    cudaError_t e = ensure_tone_levels(st);
    if (e != cudaSuccess) return e;
    unsigned long long* d = nullptr;
    if ((e = cudaMalloc(&d, 3 * sizeof(unsigned long long))) != cudaSuccess) return e;
    static uint32_t host_tbl[TONE_TABLES][TONE_BUCKETS];
    static std::mutex host_mutex;
    std::lock_guard<std::mutex> lock(host_mutex);
    if ((e = cudaMemsetAsync(d, 0, 3 * sizeof(unsigned long long), st)) == cudaSuccess) {
        k_tone_levels_verify<<<148 * 16, 256, 0, st>>>(d);
        if ((e = cudaGetLastError()) == cudaSuccess &&
            (e = cudaMemcpyAsync(mismatches, d, 3 * sizeof(unsigned long long), cudaMemcpyDeviceToHost, st)) ==
                cudaSuccess &&
            (e = cudaMemcpyFromSymbolAsync(host_tbl, g_tone_levels, sizeof(host_tbl), 0, cudaMemcpyDeviceToHost,
                                           st)) == cudaSuccess)
            e = cudaStreamSynchronize(st);
    }
    cudaFree(d);
    if (e != cudaSuccess) return e;
    for (int t = 0; t < TONE_TABLES; ++t) {
        flagged[t] = 0;
        for (uint32_t q = 0; q < TONE_BUCKETS; ++q) flagged[t] += (host_tbl[t][q] & TONE_FLAG) != 0;
    }
    return cudaSuccess;
}

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

// 16-byte alignment of the vectorised kernels' rows (cudaMalloc'd images
// are 256-byte aligned; caller buffers may not be).
static bool aligned16(const void* p) { return ((uintptr_t)p & 15u) == 0; }

// Resident blocks of 256 threads over the whole device for a kernel with
// `smem` bytes of dynamic shared memory: the grid of the grid-stride tone-map
// kernels (one wave, each block staging the tables once).  Cached per device
// and slot (kernel, type).
template <typename K>
static uint32_t wave_blocks(K kernel, uint32_t smem, int slot) {
    static std::mutex m;
    static uint32_t cache[BLOOM_NOALLOC_MAX_DEVICES][4] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= BLOOM_NOALLOC_MAX_DEVICES) return 148 * 4;
    std::lock_guard<std::mutex> lock(m);
    if (!cache[dev][slot]) {
        int sms = 0, per = 0;
        if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess ||
            cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, kernel, 256, smem) != cudaSuccess || sms <= 0 ||
            per <= 0) {
            (void)cudaGetLastError();
            return 148 * 4;
        }
        cache[dev][slot] = (uint32_t)(sms * per);
    }
    return cache[dev][slot];
}

cudaError_t launch_tonemap(const float* hdr, uint32_t npix, int type, float exposure, uint8_t* rgba, cudaStream_t st) {
    if (npix == 0) return cudaSuccess;
    cudaError_t e = ensure_tone_levels(st);
    if (e != cudaSuccess) return e;
    if (aligned16(hdr) && aligned16(rgba)) {
        const uint32_t n4 = (npix + 3) / 4;
        k_tonemap4<<<(n4 + 255) / 256, 256, 0, st>>>(hdr, npix, type, exposure, reinterpret_cast<uchar4*>(rgba));
    } else {
        k_tonemap<<<(npix + 255) / 256, 256, 0, st>>>(hdr, npix, type, exposure, reinterpret_cast<uchar4*>(rgba));
    }
    return cudaGetLastError();
}

cudaError_t launch_bloom(const float* hdr, uint32_t w, uint32_t h, const float th[4], float* scratch_half, float* out,
                         uint8_t* rgba, int type, float exposure, cudaStream_t st) {
    const uint32_t w2 = w / 2, h2 = h / 2;
    const float4 t4 = make_float4(th[0], th[1], th[2], th[3]);
    const uint32_t n2 = w2 * h2, n = w * h;
    if (rgba) {
        cudaError_t e = ensure_tone_levels(st);
        if (e != cudaSuccess) return e;
    }
    if (w % 4 == 0 && aligned16(hdr) && aligned16(scratch_half) && (rgba ? aligned16(rgba) : aligned16(out))) {
        const uint32_t pairs = (w2 / 2) * h2, quads = (w / 4) * ((h + 1) / 2);  // quad pairs of k_bloom_up4
        if (pairs) k_bloom_down4<<<(pairs + 255) / 256, 256, 0, st>>>(hdr, w, h, t4, scratch_half, w2, h2);
        if (rgba) {
            const uint32_t smem = tone_smem_bytes(type);
            uint32_t grid = wave_blocks(k_bloom_up4<true>, smem, type == 0 ? 2 : 3);
            if (grid > (quads + 255) / 256) grid = (quads + 255) / 256;
            k_bloom_up4<true><<<grid, 256, smem, st>>>(hdr, w, h, t4, scratch_half, w2, h2, nullptr,
                                                       reinterpret_cast<uchar4*>(rgba), type, exposure);
        } else {
            k_bloom_up4<false><<<(quads + 255) / 256, 256, 0, st>>>(hdr, w, h, t4, scratch_half, w2, h2, out,
                                                                   nullptr, 0, 0.0f);
        }
        return cudaGetLastError();
    }
    k_bloom_down<<<(n2 + 255) / 256, 256, 0, st>>>(hdr, w, h, t4, scratch_half, w2, h2);
    if (rgba)
        k_bloom_up<true><<<(n + 255) / 256, 256, 0, st>>>(hdr, w, h, t4, scratch_half, w2, h2, nullptr,
                                                         reinterpret_cast<uchar4*>(rgba), type, exposure);
    else
        k_bloom_up<false><<<(n + 255) / 256, 256, 0, st>>>(hdr, w, h, t4, scratch_half, w2, h2, out, nullptr, 0, 0.0f);
    return cudaGetLastError();
}

}  // namespace cupbr_b200

// Radiance-cache MLP on the fifth-generation tensor cores (tcgen05): FP16
// operands staged in shared memory, FP32 accumulators in tensor memory, one
// elected thread per CTA issuing the MMAs and committing them to an mbarrier
// that the CTA waits on (bounded: a wait that runs out of time counts an
// error and the CTA stops issuing, frees its tensor memory and returns).
//
//   k_rc_infer   persistent; 128 vertices per tile, one row per thread:
//                encode -> 6 x (MMA, tcgen05.ld, ReLU, FP16 -> smem)
//   k_rc_train   one 128-sample tile per CTA: forward keeping every layer's
//                activations in smem, relative L2 loss, backward with the
//                weight-gradient product (dY^T X, M = 128 with the rows past
//                the layer's width unused) and the input-gradient product
//                (dY W) per layer; the CTA's weight gradient goes to its own
//                slot (split-K over CTAs)
//   k_rc_adam    sums the CTA slots in a fixed order, Adam, FP16 copy
//
// Tensor-memory layout (M = 128, cta_group::1): row r of a product lives in
// lane r; warp w of the 4-warp CTA reads lanes [32w, 32w + 32).
#include "cache.hpp"

#include <algorithm>
#include <cmath>

namespace cupbr_b200 {

namespace {

constexpr uint32_t RC_W_BYTES = RC_WEIGHTS * 2;          // 47104
constexpr uint32_t RC_X0_BYTES = RC_TILE * RC_IN * 2;    // 24576
constexpr uint32_t RC_XH_BYTES = RC_TILE * RC_HID * 2;   // 16384
// The weight-gradient product reads a layer's output gradient as a 128-row
// MN-major operand although only out_l rows are real; the extra rows read up
// to 2 KB past the last batch group, which stays zero.
constexpr uint32_t RC_DY_BYTES = RC_XH_BYTES + 2048;
constexpr uint32_t RC_INFER_SMEM = RC_W_BYTES + RC_X0_BYTES + 64;
constexpr uint32_t RC_TRAIN_SMEM = RC_W_BYTES + RC_X0_BYTES + 5 * RC_XH_BYTES + RC_DY_BYTES + 64;
constexpr uint32_t RC_INFER_BLOCKS_PER_SM = 3;  // 3 x 64 tensor-memory columns, 3 x 72 KB smem
constexpr uint32_t RC_INFER_COLS = 64;
constexpr uint32_t RC_TRAIN_COLS = 256;         // [0, 64): layer output / input gradient, [128, 224): weight gradient
constexpr uint32_t RC_DW_COL = 128;
constexpr uint64_t RC_WAIT_NS = 2000000000ull;  // 2 s per tensor-core wait
constexpr float RC_GRAD_CLAMP = 2048.0f;        // |d loss / d output| per sample before the mean
constexpr float RC_GRAD_SCALE = 0.125f;         // FP16 output gradients carry this factor
constexpr float RC_HALF_MAX = 60000.0f;

// ---------------------------------------------------- primitives ---
__device__ __forceinline__ uint32_t smem_addr(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// Shared-memory matrix descriptor without swizzle (version 1: sm_100).
__device__ __forceinline__ uint64_t sdesc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
    return (uint64_t)((addr & 0x3FFFFu) >> 4) | ((uint64_t)(lbo >> 4) << 16) | ((uint64_t)(sbo >> 4) << 32) |
           (1ull << 46);
}
// Operand whose contraction runs along the columns of a tiled R x C matrix:
// core matrices 128 B apart along K, 16 C bytes apart along M / N; K step s
// covers columns [16 s, 16 s + 16).
__device__ __forceinline__ uint64_t kmajor(uint32_t base, uint32_t C, uint32_t s) {
    return sdesc(base + s * 256u, 128u, C * 16u);
}
// Operand whose contraction runs along the rows of a tiled R x C matrix:
// core matrices 16 C bytes apart along K, 128 B apart along M / N; K step s
// covers rows [16 s, 16 s + 16).
__device__ __forceinline__ uint64_t mnmajor(uint32_t base, uint32_t C, uint32_t s) {
    return sdesc(base + s * C * 32u, C * 16u, 128u);
}
// kind::f16 instruction descriptor: F16 A and B, F32 accumulator.
__device__ __forceinline__ uint32_t idesc(uint32_t M, uint32_t N, uint32_t a_mn, uint32_t b_mn) {
    return (1u << 4) | (a_mn << 15) | (b_mn << 16) | ((N >> 3) << 17) | ((M >> 4) << 24);
}
__device__ __forceinline__ void mma_f16(uint32_t d, uint64_t a, uint64_t b, uint32_t id, uint32_t acc) {
    asm volatile(
        "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n}\n" ::"r"(d),
        "l"(a), "l"(b), "r"(id), "r"(acc)
        : "memory");
}
__device__ __forceinline__ void mma_commit(uint32_t mbar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(mbar)
                 : "memory");
}
__device__ __forceinline__ void tc_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void proxy_fence() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ bool mbar_wait(uint32_t mbar, uint32_t parity, uint64_t limit_ns = RC_WAIT_NS) {
    const uint64_t t0 = gtimer();
    for (;;) {
        uint32_t ok;
        asm volatile(
            "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            "selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(ok)
            : "r"(mbar), "r"(parity)
            : "memory");
        if (ok) return true;
        if (gtimer() - t0 > limit_ns) return false;
    }
}
// A CTA whose wait for committed MMAs ran out counts itself in err[0] and
// stops issuing.  The MMAs it committed may still be writing tensor memory,
// so before the CTA frees those columns it waits once more, bounded, for that
// commit (the phase of parity `pending`); if that wait runs out too it counts
// itself in err[1]: the columns are then freed with MMAs possibly in flight
// and the host treats the cache as lost.
__device__ __forceinline__ void give_up(uint32_t mb, bool committed, uint32_t pending, uint32_t tid, uint32_t* err) {
    const bool drained = !committed || mbar_wait(mb, pending);
    const bool lost = __syncthreads_or(!drained);
    if (tid == 0) {
        atomicAdd(&err[0], 1u);
        if (lost) atomicAdd(&err[1], 1u);
    }
}
// 16 consecutive FP32 columns of this thread's lane; the wait carries the
// registers so no use is scheduled before the load has landed.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15])::"memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
// Generic-proxy smem writes -> visible to the tensor cores; tensor-memory
// reads of every thread ordered before the next MMA.
__device__ __forceinline__ void sync_for_mma() {
    proxy_fence();
    tc_before();
    __syncthreads();
    tc_after();
}
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, uint32_t cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_addr(slot)),
                 "r"(cols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
}
__device__ __forceinline__ void tmem_free(uint32_t tmem, uint32_t cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(cols));
}
__device__ __forceinline__ void mbar_init(uint64_t* mbar) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(mbar)), "r"(1));
    asm volatile("fence.mbarrier_init.release.cluster;");
}

__device__ __forceinline__ uint4 pack8(const float* v) {
    uint4 u;
    __half2 h0 = __floats2half2_rn(v[0], v[1]), h1 = __floats2half2_rn(v[2], v[3]);
    __half2 h2 = __floats2half2_rn(v[4], v[5]), h3 = __floats2half2_rn(v[6], v[7]);
    u.x = *reinterpret_cast<uint32_t*>(&h0);
    u.y = *reinterpret_cast<uint32_t*>(&h1);
    u.z = *reinterpret_cast<uint32_t*>(&h2);
    u.w = *reinterpret_cast<uint32_t*>(&h3);
    return u;
}
__device__ __forceinline__ void store8(__half* X, uint32_t row, uint32_t col, uint32_t C, const float* v) {
    *reinterpret_cast<uint4*>(X + rc_tiled(row, col, C)) = pack8(v);
}
// max(v, 0) of 8 values packed to FP16 in one conversion per pair.
__device__ __forceinline__ uint32_t relu_pack2(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.relu.f16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
__device__ __forceinline__ void store8_relu(__half* X, uint32_t row, uint32_t col, uint32_t C, const float* v) {
    *reinterpret_cast<uint4*>(X + rc_tiled(row, col, C)) =
        make_uint4(relu_pack2(v[0], v[1]), relu_pack2(v[2], v[3]), relu_pack2(v[4], v[5]), relu_pack2(v[6], v[7]));
}

// Input features of one record into row `row` of the tiled 128 x 96 input:
// [0, 72)  sin / cos (pi 2^j x) of the box-normalised position, 12 bands
//          per axis (feature 24 a + 2 j: sin, + 1: cos); band 0 from
//          sincospif, each next band by the double-angle identities
//          sin 2t = 2 s c, cos 2t = (c - s)(c + s) in FP32 (the error grows
//          ~2x per band, to ~2e-4 at band 11, under half an FP16 step)
// [72, 75) direction, [75, 78) normal, 78 roughness, [79, 82) albedo,
// 82 constant 1 (the first layer's bias), 83 remaining bounces
// min(r, 16) / 16, [84, 96) zero
__device__ __forceinline__ void rc_encode(const RcBounds& B, const float4& r0, const float4& r1, const float4& r2,
                                          const float4& r3, __half* X, uint32_t row) {
    const float pa[3] = {clampf((r0.x - B.lo.x) * B.inv_ext.x, 0.0f, 1.0f),
                         clampf((r0.y - B.lo.y) * B.inv_ext.y, 0.0f, 1.0f),
                         clampf((r0.z - B.lo.z) * B.inv_ext.z, 0.0f, 1.0f)};
#pragma unroll
    for (uint32_t a = 0; a < 3; ++a) {
        float sn, cs;
        sincospif(pa[a], &sn, &cs);
#pragma unroll
        for (uint32_t c = 0; c < 3; ++c) {
            float v[8];
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                v[2 * k] = sn;
                v[2 * k + 1] = cs;
                const float s2 = 2.0f * sn * cs;
                cs = (cs - sn) * (cs + sn);
                sn = s2;
            }
            store8(X, row, 24 * a + 8 * c, RC_IN, v);
        }
    }
    const float bounces = fminf(fmaxf(r2.w, 0.0f), RC_BOUNCE_NORM) / RC_BOUNCE_NORM;
    const float v9[8] = {r1.x, r1.y, r1.z, r2.x, r2.y, r2.z, r1.w, r3.x};
    const float v10[8] = {r3.y, r3.z, 1.0f, bounces, 0.0f, 0.0f, 0.0f, 0.0f};
    const float v11[8] = {0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f, 0.0f};
    store8(X, row, 72, RC_IN, v9);
    store8(X, row, 80, RC_IN, v10);
    store8(X, row, 88, RC_IN, v11);
}

// One layer's forward product: D[128 x out_l] = X[128 x in_l] W_l^T.
__device__ __forceinline__ void issue_forward(uint32_t l, uint32_t tmem, uint32_t xa, uint32_t wa) {
    const uint32_t K = rc_in(l), N = rc_out(l);
    const uint32_t id = idesc(128, N, 0, 0);
    const uint32_t w = wa + 2u * rc_woff(l);
    for (uint32_t s = 0; s < K / 16; ++s) mma_f16(tmem, kmajor(xa, K, s), kmajor(w, K, s), id, s > 0 ? 1u : 0u);
}

// 32 consecutive FP32 columns of this thread's lane (one wait).
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float* v) {
    uint32_t r[32];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,"
        "%16,%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31}, [%32];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
          "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
          "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
        : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;"
                 : "+r"(r[0]), "+r"(r[1]), "+r"(r[2]), "+r"(r[3]), "+r"(r[4]), "+r"(r[5]), "+r"(r[6]), "+r"(r[7]),
                   "+r"(r[8]), "+r"(r[9]), "+r"(r[10]), "+r"(r[11]), "+r"(r[12]), "+r"(r[13]), "+r"(r[14]),
                   "+r"(r[15]), "+r"(r[16]), "+r"(r[17]), "+r"(r[18]), "+r"(r[19]), "+r"(r[20]), "+r"(r[21]),
                   "+r"(r[22]), "+r"(r[23]), "+r"(r[24]), "+r"(r[25]), "+r"(r[26]), "+r"(r[27]), "+r"(r[28]),
                   "+r"(r[29]), "+r"(r[30]), "+r"(r[31])::"memory");
#pragma unroll
    for (int i = 0; i < 32; ++i) v[i] = __uint_as_float(r[i]);
}

// ReLU of a hidden layer's 64 accumulator columns -> FP16 row of X (C = 64).
__device__ __forceinline__ void hidden_epilogue(uint32_t lane_addr, __half* X, uint32_t row) {
#pragma unroll
    for (uint32_t c = 0; c < 2; ++c) {
        float v[32];
        tmem_ld32(lane_addr + 32u * c, v);
#pragma unroll
        for (int k = 0; k < 4; ++k) store8_relu(X, row, 32 * c + 8 * k, RC_HID, v + 8 * k);
    }
}

__device__ __forceinline__ void load_weights(const __half* __restrict__ w16, __half* sW) {
    const uint4* src = reinterpret_cast<const uint4*>(w16);
    uint4* dst = reinterpret_cast<uint4*>(sW);
    for (uint32_t i = threadIdx.x; i < RC_W_BYTES / 16; i += blockDim.x) dst[i] = __ldg(src + i);
}

// QUERIES = false: out[i] = network(recs[i]).  QUERIES = true: recs are
// *count cached-path queries and out is the per-path radiance, which gets
// throughput * max(network, 0) added.
template <bool QUERIES>
__global__ void __launch_bounds__(128) k_rc_infer(const __half* __restrict__ w16, RcBounds B,
                                                  const float4* __restrict__ recs, const uint32_t* __restrict__ count,
                                                  uint32_t n, float4* __restrict__ out, uint32_t* err,
                                                  uint32_t probe_ns) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __half* sW = reinterpret_cast<__half*>(smem);
    __half* sX = reinterpret_cast<__half*>(smem + RC_W_BYTES);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + RC_W_BYTES + RC_X0_BYTES);
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(mbar + 1);
    const uint32_t stride = n;  // queries: component-major records, `stride` apart
    if (QUERIES) n = min(*count, n);
    const uint32_t ntiles = (n + RC_TILE - 1) / RC_TILE;
    if (blockIdx.x >= ntiles) return;
    const uint32_t tid = threadIdx.x, warp = tid >> 5;
    load_weights(w16, sW);
    if (warp == 0) tmem_alloc(s_tmem, RC_INFER_COLS);
    if (tid == 0) mbar_init(mbar);
    sync_for_mma();
    const uint32_t tmem = *s_tmem;
    const uint32_t lane_addr = tmem + ((warp * 32u) << 16);
    const uint32_t mb = smem_addr(mbar), xa = smem_addr(sX), wa = smem_addr(sW);
    uint32_t phase = 0;
    bool failed = false, committed = false;
    if (probe_ns) {
        // Test hook (cupbr_cache_set_wait_probe): wait, before any MMA is
        // issued, on the phase of the barrier that nothing arrives on, so the
        // wait runs out after probe_ns and the CTA gives up with no
        // tensor-core work in flight.
        failed = __syncthreads_or(!mbar_wait(mb, phase, probe_ns));
    }
    // this thread's record of the next tile, loaded while the current one runs
    // (queries: and the path's radiance, which no other query of the launch touches)
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float4 p0 = z, p1 = z, p2 = z, p3 = z, p4 = z, pr = z;
    auto fetch = [&](uint32_t t) {
        const uint32_t i = t * RC_TILE + tid;
        p0 = p1 = p2 = p3 = p4 = pr = z;
        if (t < ntiles && i < n) {
            if (QUERIES) {
                const float4* r = recs + i;
                p0 = __ldg(r);
                p1 = __ldg(r + stride);
                p2 = __ldg(r + 2 * (size_t)stride);
                p3 = __ldg(r + 3 * (size_t)stride);
                p4 = __ldg(r + 4 * (size_t)stride);
                pr = out[__float_as_uint(p0.w)];
            } else {
                const float4* r = recs + (size_t)RC_REC * i;
                p0 = __ldg(r); p1 = __ldg(r + 1); p2 = __ldg(r + 2); p3 = __ldg(r + 3);
            }
        }
    };
    if (!failed) fetch(blockIdx.x);
    for (uint32_t t = blockIdx.x; t < ntiles && !failed; t += gridDim.x) {
        const uint32_t i = t * RC_TILE + tid;
        const float4 r0 = p0, r1 = p1, r2 = p2, r3 = p3, r4 = p4, rr = pr;
        fetch(t + gridDim.x);
        rc_encode(B, r0, r1, r2, r3, sX, tid);
        for (uint32_t l = 0; l < RC_LAYERS; ++l) {
            sync_for_mma();
            if (tid == 0) {
                issue_forward(l, tmem, xa, wa);
                mma_commit(mb);
            }
            const bool ok = mbar_wait(mb, phase);
            phase ^= 1u;
            if (__syncthreads_or(!ok)) {
                failed = committed = true;
                break;
            }
            tc_after();
            if (l + 1 < RC_LAYERS) {
                hidden_epilogue(lane_addr, sX, tid);
            } else {
                float v[16];
                tmem_ld16(lane_addr, v);
                if (i < n) {
                    if (QUERIES) {
                        const uint32_t pid = __float_as_uint(r0.w);
                        float4 rad = rr;
                        rad.x += r4.x * fmaxf(v[0], 0.0f);
                        rad.y += r4.y * fmaxf(v[1], 0.0f);
                        rad.z += r4.z * fmaxf(v[2], 0.0f);
                        out[pid] = rad;
                    } else {
                        out[i] = make_float4(v[0], v[1], v[2], 0.0f);
                    }
                }
            }
        }
    }
    if (failed) give_up(mb, committed, phase ^ 1u, tid, err);
    tc_before();
    __syncthreads();
    tc_after();
    if (warp == 0) tmem_free(tmem, RC_INFER_COLS);
}

__device__ __forceinline__ float block_sum128(float v, float* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31u) == 0) red[threadIdx.x >> 5] = v;
    __syncthreads();
    const float s = red[0] + red[1] + red[2] + red[3];
    __syncthreads();
    return s;
}

// Layer l's input inside the training CTA's shared memory.
__device__ __forceinline__ uint32_t x_offset(uint32_t l) {
    return RC_W_BYTES + (l == 0 ? 0u : RC_X0_BYTES + (l - 1u) * RC_XH_BYTES);
}

// Sample of training row j: direct (count == nullptr), else a stride over the
// min(*count, capacity) collected samples when there are at least `total`,
// cycling through them when there are fewer.
__device__ __forceinline__ bool sample_index(const uint32_t* count, uint32_t capacity, uint32_t total, uint32_t j,
                                             uint32_t& idx) {
    if (!count) {
        idx = j;
        return true;
    }
    const uint32_t c = min(*count, capacity);
    if (c == 0) return false;
    idx = c >= total ? (uint32_t)(((uint64_t)j * c) / total) : j % c;
    return true;
}

// One training tile of 128 samples per CTA (see the file comment).
__global__ void __launch_bounds__(128, 1) k_rc_train(const __half* __restrict__ w16, RcBounds B,
                                                     const float4* __restrict__ samples,
                                                     const uint32_t* __restrict__ count, uint32_t capacity,
                                                     uint32_t base, uint32_t total, uint32_t loss_kind,
                                                     float* __restrict__ partials, float* __restrict__ loss,
                                                     uint32_t* err) {
    extern __shared__ __align__(1024) uint8_t smem[];
    __half* sW = reinterpret_cast<__half*>(smem);
    __half* sDY = reinterpret_cast<__half*>(smem + RC_W_BYTES + RC_X0_BYTES + 5 * RC_XH_BYTES);
    uint64_t* mbar = reinterpret_cast<uint64_t*>(smem + RC_W_BYTES + RC_X0_BYTES + 5 * RC_XH_BYTES + RC_DY_BYTES);
    uint32_t* s_tmem = reinterpret_cast<uint32_t*>(mbar + 1);
    float* red = reinterpret_cast<float*>(mbar + 2);
    const uint32_t tid = threadIdx.x, warp = tid >> 5;

    load_weights(w16, sW);
    for (uint32_t i = tid; i < RC_DY_BYTES / 16; i += blockDim.x)
        reinterpret_cast<uint4*>(sDY)[i] = make_uint4(0u, 0u, 0u, 0u);
    if (warp == 0) tmem_alloc(s_tmem, RC_TRAIN_COLS);
    if (tid == 0) mbar_init(mbar);
    const float4 z = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    float4 r0 = z, r1 = z, r2 = z, r3 = z, r4 = z;
    uint32_t idx;
    if (sample_index(count, capacity, total, base + blockIdx.x * RC_TILE + tid, idx)) {
        const float4* r = samples + (size_t)RC_REC * idx;
        r0 = __ldg(r); r1 = __ldg(r + 1); r2 = __ldg(r + 2); r3 = __ldg(r + 3); r4 = __ldg(r + 4);
    }
    rc_encode(B, r0, r1, r2, r3, reinterpret_cast<__half*>(smem + x_offset(0)), tid);
    sync_for_mma();
    const uint32_t tmem = *s_tmem;
    const uint32_t lane_addr = tmem + ((warp * 32u) << 16);
    const uint32_t mb = smem_addr(mbar), wa = smem_addr(sW), dya = smem_addr(sDY), sa = smem_addr(smem);
    uint32_t phase = 0;
    bool failed = false, committed = false;

    // forward, keeping every layer's input
    float y[3] = {0.0f, 0.0f, 0.0f};
    for (uint32_t l = 0; l < RC_LAYERS && !failed; ++l) {
        if (l) sync_for_mma();
        if (tid == 0) {
            issue_forward(l, tmem, sa + x_offset(l), wa);
            mma_commit(mb);
        }
        const bool ok = mbar_wait(mb, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            failed = committed = true;
            break;
        }
        tc_after();
        if (l + 1 < RC_LAYERS) {
            hidden_epilogue(lane_addr, reinterpret_cast<__half*>(smem + x_offset(l + 1)), tid);
        } else {
            float v[16];
            tmem_ld16(lane_addr, v);
            y[0] = v[0]; y[1] = v[1]; y[2] = v[2];
        }
    }

    if (!failed) {
        // relative L2 (the prediction's square held constant) or plain L2
        const float tg[3] = {r4.x, r4.y, r4.z};
        const float w = r4.w;
        float l2 = 0.0f, g[16];
#pragma unroll
        for (int c = 0; c < 16; ++c) g[c] = 0.0f;
#pragma unroll
        for (int c = 0; c < 3; ++c) {
            const float d = y[c] - tg[c];
            const float den = loss_kind == RC_LOSS_RELATIVE ? y[c] * y[c] + 0.01f : 1.0f;
            l2 += w * d * d / den;
            g[c] = RC_GRAD_SCALE * clampf(w * 2.0f * d / den, -RC_GRAD_CLAMP, RC_GRAD_CLAMP);
        }
        store8(sDY, tid, 0, RC_OUT, g);
        store8(sDY, tid, 8, RC_OUT, g + 8);
        const float ls = block_sum128(l2, red);
        const float ws = block_sum128(w, red);
        if (tid == 0) {
            atomicAdd(&loss[0], ls);
            atomicAdd(&loss[1], ws);
        }
    }

    float* part = partials + (size_t)blockIdx.x * RC_WEIGHTS;
    for (int l = RC_LAYERS - 1; l >= 0 && !failed; --l) {
        const uint32_t K = rc_in(l), O = rc_out(l);
        sync_for_mma();
        if (tid == 0) {
            // dW_l[o][i] = sum_b dY[b][o] X_l[b][i]   (M = 128, N = in_l, K = 128 samples)
            const uint32_t idw = idesc(128, K, 1, 1);
            for (uint32_t s = 0; s < RC_TILE / 16; ++s)
                mma_f16(tmem + RC_DW_COL, mnmajor(dya, O, s), mnmajor(sa + x_offset(l), K, s), idw, s > 0 ? 1u : 0u);
            if (l > 0) {
                // dX_l[b][i] = sum_o dY[b][o] W_l[o][i]   (M = 128, N = in_l, K = out_l)
                const uint32_t idx2 = idesc(128, K, 0, 1);
                const uint32_t w = wa + 2u * rc_woff(l);
                for (uint32_t s = 0; s < O / 16; ++s)
                    mma_f16(tmem, kmajor(dya, O, s), mnmajor(w, K, s), idx2, s > 0 ? 1u : 0u);
            }
            mma_commit(mb);
        }
        const bool ok = mbar_wait(mb, phase);
        phase ^= 1u;
        if (__syncthreads_or(!ok)) {
            failed = committed = true;
            break;
        }
        tc_after();
        // weight-gradient rows: thread = output unit
        for (uint32_t c = 0; c < K / 16; ++c) {
            float v[16];
            tmem_ld16(lane_addr + RC_DW_COL + 16u * c, v);
            if (tid < O) {
                float4* p0 = reinterpret_cast<float4*>(part + rc_woff(l) + rc_tiled(tid, 16 * c, K));
                float4* p1 = reinterpret_cast<float4*>(part + rc_woff(l) + rc_tiled(tid, 16 * c + 8, K));
                p0[0] = make_float4(v[0], v[1], v[2], v[3]);
                p0[1] = make_float4(v[4], v[5], v[6], v[7]);
                p1[0] = make_float4(v[8], v[9], v[10], v[11]);
                p1[1] = make_float4(v[12], v[13], v[14], v[15]);
            }
        }
        if (l > 0) {
            // gradient of the previous layer's pre-activation: dX * [X_l > 0]
            const __half* X = reinterpret_cast<const __half*>(smem + x_offset(l));
#pragma unroll
            for (uint32_t c = 0; c < 4; ++c) {
                float v[16];
                tmem_ld16(lane_addr + 16u * c, v);
#pragma unroll
                for (int h = 0; h < 2; ++h) {
                    const uint4 u = *reinterpret_cast<const uint4*>(X + rc_tiled(tid, 16 * c + 8 * h, RC_HID));
                    const __half* xs = reinterpret_cast<const __half*>(&u);
#pragma unroll
                    for (int k = 0; k < 8; ++k) {
                        const float m = __half2float(xs[k]) > 0.0f ? 1.0f : 0.0f;
                        v[8 * h + k] = clampf(v[8 * h + k] * m, -RC_HALF_MAX, RC_HALF_MAX);
                    }
                }
                store8(sDY, tid, 16 * c, RC_HID, v);
                store8(sDY, tid, 16 * c + 8, RC_HID, v + 8);
            }
        }
    }
    if (failed) give_up(mb, committed, phase ^ 1u, tid, err);
    tc_before();
    __syncthreads();
    tc_after();
    if (warp == 0) tmem_free(tmem, RC_TRAIN_COLS);
}

// Sum of the CTA gradient slots (fixed order), mean over the weighted samples
// and the 3 channels, Adam, FP16 copy; with A.ema_decay > 0 also the weight
// average (bias-corrected by c3 = 1 - decay^step) and its FP16 copy.
// Block (32, 8): 32 weights, the slots split over 8 rows.
__global__ void k_rc_adam(RcNet N, uint32_t nparts, RcAdam A, float c1, float c2, float c3) {
    __shared__ float red[8][33];
    const uint32_t i = blockIdx.x * 32u + threadIdx.x;
    float g = 0.0f;
    if (i < RC_WEIGHTS)
        for (uint32_t p = threadIdx.y; p < nparts; p += 8u) g += N.partials[(size_t)p * RC_WEIGHTS + i];
    red[threadIdx.y][threadIdx.x] = g;
    __syncthreads();
    if (threadIdx.y != 0 || i >= RC_WEIGHTS) return;
    g = 0.0f;
    for (int y = 0; y < 8; ++y) g += red[y][threadIdx.x];
    g = g / (RC_GRAD_SCALE * 3.0f * fmaxf(N.loss[1], 1.0f));
    N.grad[i] = g;
    const float m = A.beta1 * N.adam_m[i] + (1.0f - A.beta1) * g;
    const float v = A.beta2 * N.adam_v[i] + (1.0f - A.beta2) * g * g;
    N.adam_m[i] = m;
    N.adam_v[i] = v;
    const float w = N.master[i] - A.lr * (m / c1) / (sqrtf(v / c2) + A.eps);
    N.master[i] = w;
    N.w16[i] = __float2half_rn(w);
    if (A.ema_decay > 0.0f) {
        const float e = A.ema_decay * N.ema[i] + (1.0f - A.ema_decay) * w;
        N.ema[i] = e;
        N.w16_ema[i] = __float2half_rn(e / c3);
    }
}

template <typename K>
cudaError_t set_smem(K kernel, uint32_t bytes) {
    return cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

}  // namespace

cudaError_t rc_infer(const RcNet& N, const __half* weights, const RcBounds& B, const float4* recs, uint32_t n,
                     float4* out, int num_sms, cudaStream_t st) {
    if (n == 0) return cudaSuccess;
    static cudaError_t attr = set_smem(k_rc_infer<false>, RC_INFER_SMEM);
    if (attr != cudaSuccess) return attr;
    const uint32_t tiles = (n + RC_TILE - 1) / RC_TILE;
    const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)num_sms * RC_INFER_BLOCKS_PER_SM);
    k_rc_infer<false><<<grid, 128, RC_INFER_SMEM, st>>>(weights, B, recs, nullptr, n, out, N.err,
                                                         N.wait_probe_ns);
    return cudaGetLastError();
}

cudaError_t rc_infer_queries(const RcNet& N, const __half* weights, const RcBounds& B, const float4* recs,
                             const uint32_t* count, uint32_t capacity, float4* radiance, int num_sms, cudaStream_t st) {
    if (capacity == 0) return cudaSuccess;
    static cudaError_t attr = set_smem(k_rc_infer<true>, RC_INFER_SMEM);
    if (attr != cudaSuccess) return attr;
    const uint32_t tiles = (capacity + RC_TILE - 1) / RC_TILE;
    const uint32_t grid = std::min<uint32_t>(tiles, (uint32_t)num_sms * RC_INFER_BLOCKS_PER_SM);
    k_rc_infer<true><<<grid, 128, RC_INFER_SMEM, st>>>(weights, B, recs, count, capacity, radiance, N.err,
                                                        N.wait_probe_ns);
    return cudaGetLastError();
}

cudaError_t rc_train_step(const RcNet& N, const RcBounds& B, const float4* samples, const uint32_t* count,
                          uint32_t capacity, uint32_t base, uint32_t total, uint32_t n, const RcAdam& A,
                          cudaStream_t st) {
    if (n == 0 || n % RC_TILE != 0 || n / RC_TILE > N.partial_ctas) return cudaErrorInvalidValue;
    static cudaError_t attr = set_smem(k_rc_train, RC_TRAIN_SMEM);
    if (attr != cudaSuccess) return attr;
    cudaError_t e = cudaMemsetAsync(N.loss, 0, 2 * sizeof(float), st);
    if (e != cudaSuccess) return e;
    const uint32_t ctas = n / RC_TILE;
    k_rc_train<<<ctas, 128, RC_TRAIN_SMEM, st>>>(N.w16, B, samples, count, capacity, base, total, A.loss,
                                                 N.partials, N.loss, N.err);
    const double c1 = 1.0 - std::pow((double)A.beta1, (double)A.step);
    const double c2 = 1.0 - std::pow((double)A.beta2, (double)A.step);
    const double c3 = A.ema_decay > 0.0f ? 1.0 - std::pow((double)A.ema_decay, (double)A.step) : 1.0;
    k_rc_adam<<<(RC_WEIGHTS + 31) / 32, dim3(32, 8), 0, st>>>(N, ctas, A, (float)c1, (float)c2, (float)c3);
    return cudaGetLastError();
}

}  // namespace cupbr_b200

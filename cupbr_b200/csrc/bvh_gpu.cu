// Device build of the binned-SAH BVH (see bvh_gpu.hpp).  The split rules
// are those of TypeBuilder::build in bvh_build.cpp, evaluated with the same
// float operations (this file is compiled with -fmad=false, the host file
// with -ffp-contract=off):
//   * centroid 0.5 * (lo + hi); 16 bins per axis over the centroid bounds,
//     bin = min(15, (int)((c - lo) * (16 / extent))), axes of zero extent
//     skipped;
//   * SAH sweep right-to-left for the right areas, left-to-right for the
//     costs, first strictly smaller cost wins (axis 0, 1, 2; split 1..15);
//   * leaf when n <= 1, or n <= max_leaf and the split is not cheaper than
//     n primitive tests; below depth 44, or with no SAH split, the object
//     median on the widest centroid axis by (centroid, id);
//   * a leaf lists its primitives in ascending id order.
// Bounds are exact minima / maxima, so the order in which primitives are
// binned or partitioned changes nothing.
#include "bvh_gpu.hpp"
#include "dev_alloc.hpp"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <numeric>

namespace cupbr_b200 {

namespace {

constexpr int NB = 16;                 // bins per axis
constexpr uint32_t SAH_DEPTH = 44;     // from this depth on: object median
constexpr uint32_t SMALL = 960;        // subtrees up to this size: one CTA each (shared memory < 48 KB)
constexpr uint32_t CHUNK = 8192;       // primitives per binning block of a large node
constexpr int BW = 13;                 // words per large-node bin: box lo/hi, centroid lo/hi, count
constexpr int LB_WORDS = 3 * NB * BW;  // bins of one large node
constexpr int SB_THREADS = 256;
constexpr uint32_t WARP_SUBTREE = 32;   // subtrees up to this size: one warp each
constexpr uint32_t ORD_PINF = 0xff800000u;  // ord(+inf)
constexpr uint32_t ORD_NINF = 0x007fffffu;  // ord(-inf)

// Binary node; left < 0 marks a leaf over slots [start, start + count).
struct DNode {
    float lo[3], hi[3];
    int32_t left, right;
    uint32_t start, count;
};

struct LTask {
    uint32_t node, b, e, depth;
    float clo[3], chi[3];
    uint32_t chunk0, nchunk;
};
struct LChunk {
    uint32_t task, begin, end;
};
struct LResult {
    int32_t axis, split;  // axis -1: no SAH split (the host takes the median)
    uint32_t mid, left;   // first position of the right child; left child node
    float clo[2][3], chi[2][3];  // centroid bounds of the two children
};
struct STask {
    uint32_t node, b, e, depth;
};
// 4-wide node under construction: binary source node, collapsed children,
// and for inner children the index of their own W4 entry.
struct W4 {
    int32_t src, n, depth, pad;
    int32_t child[4];
    int32_t c4[4];
};

__device__ __forceinline__ uint32_t ord(float f) {
    const uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float unord(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7fffffffu) : ~u);
}

__host__ __device__ __forceinline__ float harea(const float lo[3], const float hi[3]) {
    const float dx = hi[0] - lo[0], dy = hi[1] - lo[1], dz = hi[2] - lo[2];
    if (dx < 0 || dy < 0 || dz < 0) return 0.0f;
    return dx * dy + dy * dz + dz * dx;
}

__device__ __forceinline__ int bin_of(float c, float lo, float scale) {
    return min(NB - 1, (int)((c - lo) * scale));
}

// The SAH sweep of bvh_build.cpp over per-axis bins given as float boxes
// and counts (blo/bhi[ax][s][3], cnt[ax][s]); axes with ext[ax] <= 0 skipped.
__device__ void sah_sweep(const float (*blo)[NB][3], const float (*bhi)[NB][3], const uint32_t (*cnt)[NB],
                          const float ext[3], float& best_cost, int& best_axis, int& best_split) {
    best_cost = __int_as_float(0x7f800000);
    best_axis = -1;
    best_split = -1;
    for (int ax = 0; ax < 3; ++ax) {
        if (!(ext[ax] > 0.0f)) continue;
        float right_area[NB];
        uint32_t right_cnt[NB];
        float alo[3] = {INFINITY, INFINITY, INFINITY}, ahi[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t c = 0;
        for (int s = NB - 1; s > 0; --s) {
            for (int k = 0; k < 3; ++k) { alo[k] = fminf(alo[k], blo[ax][s][k]); ahi[k] = fmaxf(ahi[k], bhi[ax][s][k]); }
            c += cnt[ax][s];
            right_area[s] = harea(alo, ahi);
            right_cnt[s] = c;
        }
        float llo[3] = {INFINITY, INFINITY, INFINITY}, lhi[3] = {-INFINITY, -INFINITY, -INFINITY};
        uint32_t lc = 0;
        for (int s = 1; s < NB; ++s) {
            for (int k = 0; k < 3; ++k) { llo[k] = fminf(llo[k], blo[ax][s - 1][k]); lhi[k] = fmaxf(lhi[k], bhi[ax][s - 1][k]); }
            lc += cnt[ax][s - 1];
            if (lc == 0 || right_cnt[s] == 0) continue;
            const float cost = harea(llo, lhi) * (float)lc + right_area[s] * (float)right_cnt[s];
            if (cost < best_cost) { best_cost = cost; best_axis = ax; best_split = s; }
        }
    }
}

// The same sweep for one axis by one warp, lane s holding bin s: the right
// boxes / counts are suffix scans, the left ones prefix scans (min / max and
// integer sums, exact in any order), and the first strictly smallest cost
// is the smallest (cost, split) pair.  bins: [NB][7] ordered words (box lo,
// box hi, count).  Returns cost INF when no split has both sides non-empty.
__device__ void sah_sweep_warp(const uint32_t (*bins)[7], float& best_cost, int& best_split) {
    const unsigned full = 0xffffffffu;
    const int lane = (int)(threadIdx.x & 31u);
    const float INF = __int_as_float(0x7f800000);
    float lo[3], hi[3];
    uint32_t c = 0;
    for (int k = 0; k < 3; ++k) { lo[k] = INF; hi[k] = -INF; }
    if (lane < NB) {
        for (int k = 0; k < 3; ++k) { lo[k] = unord(bins[lane][k]); hi[k] = unord(bins[lane][3 + k]); }
        c = bins[lane][6];
    }
    float rlo[3], rhi[3], plo[3], phi[3];
    uint32_t rc = c, pc = c;
    for (int k = 0; k < 3; ++k) { rlo[k] = plo[k] = lo[k]; rhi[k] = phi[k] = hi[k]; }
    for (int o = 1; o < NB; o <<= 1) {
        const bool down = lane + o < NB, up = lane >= o;
        for (int k = 0; k < 3; ++k) {
            const float dl = __shfl_down_sync(full, rlo[k], o), dh = __shfl_down_sync(full, rhi[k], o);
            const float ul = __shfl_up_sync(full, plo[k], o), uh = __shfl_up_sync(full, phi[k], o);
            if (down) { rlo[k] = fminf(rlo[k], dl); rhi[k] = fmaxf(rhi[k], dh); }
            if (up) { plo[k] = fminf(plo[k], ul); phi[k] = fmaxf(phi[k], uh); }
        }
        const uint32_t dc = __shfl_down_sync(full, rc, o), uc = __shfl_up_sync(full, pc, o);
        if (down) rc += dc;
        if (up) pc += uc;
    }
    // split s: left = bins 0..s-1 (the prefix at s - 1), right = bins s..15
    float llo[3], lhi[3];
    for (int k = 0; k < 3; ++k) { llo[k] = __shfl_up_sync(full, plo[k], 1); lhi[k] = __shfl_up_sync(full, phi[k], 1); }
    const uint32_t lc = __shfl_up_sync(full, pc, 1);
    float cost = INF;
    int split = NB;
    if (lane >= 1 && lane < NB && lc != 0 && rc != 0) {
        const float cc = harea(llo, lhi) * (float)lc + harea(rlo, rhi) * (float)rc;
        if (cc < INF) { cost = cc; split = lane; }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const float oc = __shfl_xor_sync(full, cost, o);
        const int os = __shfl_xor_sync(full, split, o);
        if (oc < cost || (oc == cost && os < split)) { cost = oc; split = os; }
    }
    best_cost = cost;
    best_split = split;
}

__host__ __device__ __forceinline__ int widest_axis(const float clo[3], const float chi[3]) {
    const float w0 = chi[0] - clo[0], w1 = chi[1] - clo[1], w2 = chi[2] - clo[2];
    if (w1 > w0 && w1 >= w2) return 1;
    if (w2 > w0 && w2 > w1) return 2;
    return 0;
}

// Box of primitive i in the PrimBox array (6 floats: lo xyz, hi xyz; 8-byte
// aligned, read as three float2).
__device__ __forceinline__ void load_box(const float2* __restrict__ pb, uint32_t i, float lo[3], float hi[3]) {
    const float2 a = __ldg(&pb[3 * (size_t)i]), b = __ldg(&pb[3 * (size_t)i + 1]), c = __ldg(&pb[3 * (size_t)i + 2]);
    lo[0] = a.x; lo[1] = a.y; lo[2] = b.x;
    hi[0] = b.y; hi[1] = c.x; hi[2] = c.y;
}

__global__ void k_iota(uint32_t* idx, uint32_t n) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) idx[i] = i;
}

// Box and centroid bounds of all primitives of one type (ordered words:
// box lo[3], box hi[3], centroid lo[3], centroid hi[3]).
__global__ void k_root_bounds(const float2* __restrict__ pb, uint32_t n, uint32_t* out) {
    float v[12];
    for (int k = 0; k < 3; ++k) { v[k] = v[6 + k] = INFINITY; v[3 + k] = v[9 + k] = -INFINITY; }
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float lo[3], hi[3];
        load_box(pb, i, lo, hi);
        for (int k = 0; k < 3; ++k) {
            const float c = 0.5f * (lo[k] + hi[k]);
            v[k] = fminf(v[k], lo[k]);
            v[3 + k] = fmaxf(v[3 + k], hi[k]);
            v[6 + k] = fminf(v[6 + k], c);
            v[9 + k] = fmaxf(v[9 + k], c);
        }
    }
    for (int k = 0; k < 12; ++k) {
        const bool is_min = (k % 6) < 3;
        float x = v[k];
        for (int o = 16; o > 0; o >>= 1) {
            const float y = __shfl_xor_sync(0xffffffffu, x, o);
            x = is_min ? fminf(x, y) : fmaxf(x, y);
        }
        if ((threadIdx.x & 31u) == 0) {
            if (is_min) atomicMin(&out[k], ord(x));
            else atomicMax(&out[k], ord(x));
        }
    }
}

__global__ void k_init_bins(uint32_t* bins, uint32_t words) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= words) return;
    const uint32_t w = i % BW;
    bins[i] = w == 12 ? 0u : ((w < 3 || (w >= 6 && w < 9)) ? ORD_PINF : ORD_NINF);
}

// Bins the primitives of one chunk of a large node along all three axes
// (shared-memory atomics), then merges into the node's bins; the chunk's
// own per-bin counts are kept for the partition offsets.
__global__ void __launch_bounds__(256) k_bin_large(const LTask* __restrict__ tasks, const LChunk* __restrict__ chunks,
                                                   const uint32_t* __restrict__ idx, const float2* __restrict__ pb,
                                                   uint32_t* __restrict__ bins, uint32_t* __restrict__ chunk_cnt) {
    __shared__ uint32_t sb[LB_WORDS];
    const LChunk C = chunks[blockIdx.x];
    const LTask T = tasks[C.task];
    for (int i = threadIdx.x; i < LB_WORDS; i += blockDim.x) {
        const int w = i % BW;
        sb[i] = w == 12 ? 0u : ((w < 3 || (w >= 6 && w < 9)) ? ORD_PINF : ORD_NINF);
    }
    float scale[3];
    bool use[3];
    for (int k = 0; k < 3; ++k) {
        const float ext = T.chi[k] - T.clo[k];
        use[k] = ext > 0.0f;
        scale[k] = (float)NB / ext;
    }
    __syncthreads();
    for (uint32_t p = C.begin + threadIdx.x; p < C.end; p += blockDim.x) {
        const uint32_t pi = idx[p];
        float lo[3], hi[3];
        load_box(pb, pi, lo, hi);
        const float c[3] = {0.5f * (lo[0] + hi[0]), 0.5f * (lo[1] + hi[1]), 0.5f * (lo[2] + hi[2])};
        for (int ax = 0; ax < 3; ++ax) {
            if (!use[ax]) continue;
            uint32_t* w = sb + (ax * NB + bin_of(c[ax], T.clo[ax], scale[ax])) * BW;
            for (int k = 0; k < 3; ++k) {
                atomicMin(&w[k], ord(lo[k]));
                atomicMax(&w[3 + k], ord(hi[k]));
                atomicMin(&w[6 + k], ord(c[k]));
                atomicMax(&w[9 + k], ord(c[k]));
            }
            atomicAdd(&w[12], 1u);
        }
    }
    __syncthreads();
    uint32_t* gb = bins + (size_t)C.task * LB_WORDS;
    for (int i = threadIdx.x; i < 3 * NB; i += blockDim.x) chunk_cnt[(size_t)blockIdx.x * 3 * NB + i] = sb[i * BW + 12];
    for (int i = threadIdx.x; i < LB_WORDS; i += blockDim.x) {
        const int w = i % BW;
        if (sb[(i / BW) * BW + 12] == 0) continue;  // empty bin
        if (w == 12) atomicAdd(&gb[i], sb[i]);
        else if (w < 3 || (w >= 6 && w < 9)) atomicMin(&gb[i], sb[i]);
        else atomicMax(&gb[i], sb[i]);
    }
}

// One thread per large node: the SAH split from its bins, the two children
// (boxes written, nodes allocated) and each chunk's offsets into them.
__global__ void k_split_large(const LTask* __restrict__ tasks, uint32_t ntasks, const uint32_t* __restrict__ bins,
                              const uint32_t* __restrict__ chunk_cnt, DNode* __restrict__ nodes,
                              uint32_t* __restrict__ node_ctr, uint32_t node_cap, LResult* __restrict__ res,
                              uint32_t* __restrict__ chunk_off, uint32_t* __restrict__ err) {
    const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= ntasks) return;
    const LTask T = tasks[t];
    const uint32_t* gb = bins + (size_t)t * LB_WORDS;
    float blo[3][NB][3], bhi[3][NB][3];
    uint32_t cnt[3][NB];
    float ext[3];
    for (int ax = 0; ax < 3; ++ax) {
        ext[ax] = T.chi[ax] - T.clo[ax];
        for (int s = 0; s < NB; ++s) {
            const uint32_t* w = gb + (ax * NB + s) * BW;
            for (int k = 0; k < 3; ++k) { blo[ax][s][k] = unord(w[k]); bhi[ax][s][k] = unord(w[3 + k]); }
            cnt[ax][s] = w[12];
        }
    }
    LResult R{};
    R.axis = -1;
    if (T.depth < SAH_DEPTH) {
        float best_cost;
        int best_axis, best_split;
        sah_sweep(blo, bhi, cnt, ext, best_cost, best_axis, best_split);
        R.axis = best_axis;
        R.split = best_split;
    }
    if (R.axis < 0) {  // object median: taken by the host
        res[t] = R;
        return;
    }
    const int ax = R.axis, sp = R.split;
    uint32_t lc = 0;
    float box[2][6];
    for (int h = 0; h < 2; ++h)
        for (int k = 0; k < 3; ++k) {
            box[h][k] = INFINITY; box[h][3 + k] = -INFINITY;
            R.clo[h][k] = INFINITY; R.chi[h][k] = -INFINITY;
        }
    for (int s = 0; s < NB; ++s) {
        if (cnt[ax][s] == 0) continue;
        const int h = s < sp ? 0 : 1;
        if (h == 0) lc += cnt[ax][s];
        const uint32_t* w = gb + (ax * NB + s) * BW;
        for (int k = 0; k < 3; ++k) {
            box[h][k] = fminf(box[h][k], unord(w[k]));
            box[h][3 + k] = fmaxf(box[h][3 + k], unord(w[3 + k]));
            R.clo[h][k] = fminf(R.clo[h][k], unord(w[6 + k]));
            R.chi[h][k] = fmaxf(R.chi[h][k], unord(w[9 + k]));
        }
    }
    R.mid = T.b + lc;
    const uint32_t l = atomicAdd(node_ctr, 2u);
    if (l + 2 > node_cap) {
        atomicAdd(err, 1u);
        R.axis = -2;
        res[t] = R;
        return;
    }
    R.left = l;
    for (int h = 0; h < 2; ++h) {
        DNode c;
        for (int k = 0; k < 3; ++k) { c.lo[k] = box[h][k]; c.hi[k] = box[h][3 + k]; }
        c.left = c.right = -1;
        c.start = c.count = 0;
        nodes[l + h] = c;
    }
    nodes[T.node].left = (int32_t)l;
    nodes[T.node].right = (int32_t)(l + 1);
    // chunk offsets: chunk c's left primitives go to [b + lo, ...), its
    // right ones to [mid + ro, ...)
    uint32_t lo = 0, ro = 0;
    for (uint32_t c = 0; c < T.nchunk; ++c) {
        const uint32_t* cc = chunk_cnt + (size_t)(T.chunk0 + c) * 3 * NB + ax * NB;
        uint32_t cl = 0, cr = 0;
        for (int s = 0; s < NB; ++s) (s < sp ? cl : cr) += cc[s];
        chunk_off[2 * (T.chunk0 + c)] = lo;
        chunk_off[2 * (T.chunk0 + c) + 1] = ro;
        lo += cl;
        ro += cr;
    }
    res[t] = R;
}

// Scatters one chunk's primitives to the two children's ranges (the order
// inside a range does not matter).
__global__ void __launch_bounds__(256) k_partition_large(const LTask* __restrict__ tasks,
                                                         const LChunk* __restrict__ chunks,
                                                         const LResult* __restrict__ res,
                                                         const uint32_t* __restrict__ chunk_off,
                                                         const uint32_t* __restrict__ idx,
                                                         const float2* __restrict__ pb, uint32_t* __restrict__ tmp) {
    __shared__ uint32_t s_n[2];
    const LChunk C = chunks[blockIdx.x];
    const LResult R = res[C.task];
    if (R.axis < 0) return;
    const LTask T = tasks[C.task];
    if (threadIdx.x < 2) s_n[threadIdx.x] = 0;
    __syncthreads();
    const int ax = R.axis;
    const float scale = (float)NB / (T.chi[ax] - T.clo[ax]);
    const uint32_t lbase = T.b + chunk_off[2 * blockIdx.x], rbase = R.mid + chunk_off[2 * blockIdx.x + 1];
    for (uint32_t p = C.begin + threadIdx.x; p < C.end; p += blockDim.x) {
        const uint32_t pi = idx[p];
        float lo[3], hi[3];
        load_box(pb, pi, lo, hi);
        const bool left = bin_of(0.5f * (lo[ax] + hi[ax]), T.clo[ax], scale) < R.split;
        const uint32_t r = atomicAdd(&s_n[left ? 0 : 1], 1u);
        tmp[(left ? lbase : rbase) + r] = pi;
    }
}

__global__ void k_copy_range(const LChunk* __restrict__ chunks, const LResult* __restrict__ res,
                             const uint32_t* __restrict__ tmp, uint32_t* __restrict__ idx) {
    const LChunk C = chunks[blockIdx.x];
    if (res[C.task].axis < 0) return;
    for (uint32_t p = C.begin + threadIdx.x; p < C.end; p += blockDim.x) idx[p] = tmp[p];
}

// Block-wide min (first 6 of 12 values: box lo, centroid lo) / max reduction.
__device__ __forceinline__ void block_bounds(float v[12], float (*red)[12]) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    for (int k = 0; k < 12; ++k) {
        const bool is_min = (k % 6) < 3;
        float x = v[k];
        for (int o = 16; o > 0; o >>= 1) {
            const float y = __shfl_xor_sync(0xffffffffu, x, o);
            x = is_min ? fminf(x, y) : fmaxf(x, y);
        }
        if (lane == 0) red[warp][k] = x;
    }
    __syncthreads();
    for (int k = 0; k < 12; ++k) {
        const bool is_min = (k % 6) < 3;
        float x = red[0][k];
        for (int w = 1; w < SB_THREADS / 32; ++w) x = is_min ? fminf(x, red[w][k]) : fmaxf(x, red[w][k]);
        v[k] = x;
    }
    __syncthreads();
}

// One warp builds the whole subtree of a node of at most 32 primitives, lane
// i holding the node's i-th primitive: the decisions of the CTA loop below
// (bounds by shuffles, one axis binned at a time into the warp's bins, the
// same SAH sweep, leaf rule, partition by ballot ranks, object median by
// (centroid, id) ranks) without block barriers.  stack / depth: the warp's
// 32 entries of pending nodes.  Returns false when the node array is full.
__device__ bool warp_subtree(uint2 root, uint32_t root_depth, const float (*s_box)[6], const uint32_t* s_id,
                             uint16_t* s_perm, uint2* stack, uint16_t* sdepth, uint32_t (*bins)[7],
                             DNode* __restrict__ nodes, uint32_t* __restrict__ node_ctr, uint32_t node_cap,
                             uint32_t slot_base, int max_leaf, float trav_cost) {
    const unsigned full = 0xffffffffu;
    const uint32_t lane = threadIdx.x & 31u;
    const float INF = __int_as_float(0x7f800000);
    if (lane == 0) {
        stack[0] = root;
        sdepth[0] = (uint16_t)root_depth;
    }
    __syncwarp();
    int sp = 1;
    while (sp > 0) {
        --sp;
        const uint2 E = stack[sp];
        const uint32_t depth = sdepth[sp];
        __syncwarp();
        const uint32_t node = E.x, lb = E.y & 0xffffu, le = E.y >> 16, n = le - lb;
        const bool act = lane < n;
        const uint16_t j = act ? s_perm[lb + lane] : (uint16_t)0;
        float lo[3], hi[3], c[3];
        for (int k = 0; k < 3; ++k) {
            lo[k] = act ? s_box[j][k] : INF;
            hi[k] = act ? s_box[j][3 + k] : -INF;
            c[k] = 0.5f * (s_box[j][k] + s_box[j][3 + k]);
        }
        float v[12];
        for (int k = 0; k < 3; ++k) {
            v[k] = lo[k];
            v[3 + k] = hi[k];
            v[6 + k] = act ? c[k] : INF;
            v[9 + k] = act ? c[k] : -INF;
        }
        for (int k = 0; k < 12; ++k) {
            const bool is_min = (k % 6) < 3;
            for (int o = 16; o > 0; o >>= 1) {
                const float y = __shfl_xor_sync(full, v[k], o);
                v[k] = is_min ? fminf(v[k], y) : fmaxf(v[k], y);
            }
        }
        const float* clo = v + 6;
        const float* chi = v + 9;
        float ext[3], scale[3];
        for (int k = 0; k < 3; ++k) {
            ext[k] = chi[k] - clo[k];
            scale[k] = (float)NB / ext[k];
        }
        int axis = -1, split = -1;
        bool leaf = false;
        if (n <= 1) {
            leaf = true;
        } else {
            float best_cost = INF;
            if (depth < SAH_DEPTH) {
                for (int ax = 0; ax < 3; ++ax) {
                    if (!(ext[ax] > 0.0f)) continue;
                    for (uint32_t i = lane; i < NB * 7; i += 32) {
                        const uint32_t w = i % 7;
                        (&bins[0][0])[i] = w == 6 ? 0u : (w < 3 ? ORD_PINF : ORD_NINF);
                    }
                    __syncwarp();
                    if (act) {
                        uint32_t* w = bins[bin_of(c[ax], clo[ax], scale[ax])];
                        for (int k = 0; k < 3; ++k) {
                            atomicMin(&w[k], ord(lo[k]));
                            atomicMax(&w[3 + k], ord(hi[k]));
                        }
                        atomicAdd(&w[6], 1u);
                    }
                    __syncwarp();
                    float cst;
                    int sp_ax;
                    sah_sweep_warp(bins, cst, sp_ax);
                    if (cst < best_cost) { best_cost = cst; axis = ax; split = sp_ax; }
                    __syncwarp();
                }
            }
            const float parent_area = harea(v, v + 3);
            const float leaf_cost = (float)n;
            const float split_cost =
                axis >= 0 ? trav_cost + (parent_area > 0 ? best_cost / parent_area : (float)n) : INF;
            if (n <= (uint32_t)max_leaf && !(split_cost < leaf_cost)) leaf = true;
        }
        if (leaf) {
            if (lane == 0) {
                // ascending primitive ids
                for (uint32_t i = lb + 1; i < le; ++i) {
                    const uint16_t x = s_perm[i];
                    uint32_t q = i;
                    while (q > lb && s_id[s_perm[q - 1]] > s_id[x]) { s_perm[q] = s_perm[q - 1]; --q; }
                    s_perm[q] = x;
                }
                DNode d;
                for (int k = 0; k < 3; ++k) { d.lo[k] = v[k]; d.hi[k] = v[3 + k]; }
                d.left = d.right = -1;
                d.start = slot_base + lb;
                d.count = n;
                nodes[node] = d;
            }
            __syncwarp();
            continue;
        }
        uint32_t pos, mid;
        const unsigned below = (1u << lane) - 1u;
        if (axis >= 0) {
            const bool left = act && bin_of(c[axis], clo[axis], scale[axis]) < split;
            const unsigned lm = __ballot_sync(full, left), am = __ballot_sync(full, act);
            const uint32_t nl = (uint32_t)__popc(lm);
            pos = left ? lb + (uint32_t)__popc(lm & below) : lb + nl + (uint32_t)__popc(am & ~lm & below);
            mid = lb + nl;
        } else {
            // object median on the widest centroid axis by (centroid, id)
            const int ax = widest_axis(clo, chi);
            const float ca = c[ax];
            const uint32_t id = act ? s_id[j] : 0xffffffffu;
            uint32_t rank = 0;
            for (uint32_t q = 0; q < n; ++q) {
                const float cq = __shfl_sync(full, ca, (int)q);
                const uint32_t iq = __shfl_sync(full, id, (int)q);
                rank += (cq < ca || (cq == ca && iq < id)) ? 1u : 0u;
            }
            pos = lb + rank;
            mid = lb + n / 2;
        }
        __syncwarp();
        if (act) s_perm[pos] = j;
        int ok = 1;
        if (lane == 0) {
            const uint32_t l = atomicAdd(node_ctr, 2u);
            if (l + 2 > node_cap || sp + 2 > (int)WARP_SUBTREE) {
                ok = 0;
            } else {
                DNode d;
                for (int k = 0; k < 3; ++k) { d.lo[k] = v[k]; d.hi[k] = v[3 + k]; }
                d.left = (int32_t)l;
                d.right = (int32_t)(l + 1);
                d.start = d.count = 0;
                nodes[node] = d;
                stack[sp] = make_uint2(l + 1, mid | (le << 16));
                sdepth[sp] = (uint16_t)(depth + 1);
                stack[sp + 1] = make_uint2(l, lb | (mid << 16));
                sdepth[sp + 1] = (uint16_t)(depth + 1);
            }
        }
        ok = __shfl_sync(full, ok, 0);
        __syncwarp();
        if (!ok) return false;
        sp += 2;
    }
    return true;
}

// One CTA builds the whole subtree of a node of at most SMALL primitives in
// shared memory: nodes of more than 32 primitives depth first by the whole
// block (an explicit stack of pending nodes), the subtrees of at most 32 set
// aside and then built one per warp (warp_subtree).
__global__ void __launch_bounds__(SB_THREADS, 4) k_build_small(const STask* __restrict__ tasks,
                                                            uint32_t* __restrict__ idx, const float2* __restrict__ pb,
                                                            DNode* __restrict__ nodes, uint32_t* __restrict__ node_ctr,
                                                            uint32_t node_cap, uint32_t slot_off, int max_leaf,
                                                            float trav_cost, uint32_t* __restrict__ err) {
    __shared__ float s_box[SMALL][6];
    __shared__ uint32_t s_id[SMALL];
    __shared__ uint16_t s_perm[SMALL], s_tmp[SMALL];
    __shared__ uint2 s_stack[SMALL];  // pending nodes: (node, lb | le << 16)
    __shared__ uint16_t s_depth[SMALL];
    __shared__ uint32_t s_bins[3][NB][7];
    __shared__ float s_red[SB_THREADS / 32][12];
    __shared__ int s_pick[3];  // axis, split, leaf
    __shared__ float s_axc[3];  // best cost per axis
    __shared__ int s_axs[3];    // and its split
    __shared__ uint32_t s_cnt[2];
    __shared__ int s_fail;
    __shared__ uint32_t s_wbins[SB_THREADS / 32][NB][7];  // one axis of bins per warp (phase 2)
    __shared__ uint2 s_wstack[SB_THREADS / 32][WARP_SUBTREE];  // pending nodes per warp (phase 2)
    __shared__ uint16_t s_wdepth[SB_THREADS / 32][WARP_SUBTREE];
    __shared__ uint32_t s_list_n, s_list_next;           // subtrees of <= 32 set aside, at the top of s_stack
    __shared__ int s_push;                                // stack entries the last split pushed

    const STask T = tasks[blockIdx.x];
    const uint32_t n0 = T.e - T.b;
    for (uint32_t i = threadIdx.x; i < n0; i += blockDim.x) {
        const uint32_t pi = idx[T.b + i];
        float lo[3], hi[3];
        load_box(pb, pi, lo, hi);
        s_id[i] = pi;
        for (int k = 0; k < 3; ++k) { s_box[i][k] = lo[k]; s_box[i][3 + k] = hi[k]; }
        s_perm[i] = (uint16_t)i;
    }
    // phase 1: nodes of more than 32 primitives, depth first by the block;
    // smaller ones go to the list at the top of s_stack (stack + list never
    // hold more entries than primitives: list entries hold >= 1 primitive
    // each, pending stack entries > 32)
    const bool root_small = n0 <= WARP_SUBTREE;
    if (threadIdx.x == 0) {
        const uint32_t at = root_small ? SMALL - 1 : 0u;
        s_stack[at] = make_uint2(T.node, 0u | (n0 << 16));
        s_depth[at] = (uint16_t)T.depth;
        s_list_n = root_small ? 1u : 0u;
        s_list_next = 0;
        s_fail = 0;
    }
    __syncthreads();
    int sp = root_small ? 0 : 1;
    while (sp > 0) {
        --sp;
        const uint2 E = s_stack[sp];
        const uint32_t depth = s_depth[sp];
        const uint32_t node = E.x, lb = E.y & 0xffffu, le = E.y >> 16, n = le - lb;
        // box and centroid bounds of [lb, le)
        float v[12];
        for (int k = 0; k < 3; ++k) { v[k] = v[6 + k] = INFINITY; v[3 + k] = v[9 + k] = -INFINITY; }
        for (uint32_t i = lb + threadIdx.x; i < le; i += blockDim.x) {
            const float* bx = s_box[s_perm[i]];
            for (int k = 0; k < 3; ++k) {
                const float c = 0.5f * (bx[k] + bx[3 + k]);
                v[k] = fminf(v[k], bx[k]);
                v[3 + k] = fmaxf(v[3 + k], bx[3 + k]);
                v[6 + k] = fminf(v[6 + k], c);
                v[9 + k] = fmaxf(v[9 + k], c);
            }
        }
        block_bounds(v, s_red);  // ends with a barrier: the stack entry has been read by all
        const float* clo = v + 6;
        const float* chi = v + 9;
        float ext[3], scale[3];
        for (int k = 0; k < 3; ++k) {
            ext[k] = chi[k] - clo[k];
            scale[k] = (float)NB / ext[k];
        }
        // split decision
        if (n > 1 && depth < SAH_DEPTH) {
            for (uint32_t i = threadIdx.x; i < 3 * NB * 7; i += blockDim.x) {
                const uint32_t w = i % 7;
                (&s_bins[0][0][0])[i] = w == 6 ? 0u : (w < 3 ? ORD_PINF : ORD_NINF);
            }
            __syncthreads();
            for (uint32_t i = lb + threadIdx.x; i < le; i += blockDim.x) {
                const float* bx = s_box[s_perm[i]];
                for (int ax = 0; ax < 3; ++ax) {
                    if (!(ext[ax] > 0.0f)) continue;
                    uint32_t* w = s_bins[ax][bin_of(0.5f * (bx[ax] + bx[3 + ax]), clo[ax], scale[ax])];
                    for (int k = 0; k < 3; ++k) {
                        atomicMin(&w[k], ord(bx[k]));
                        atomicMax(&w[3 + k], ord(bx[3 + k]));
                    }
                    atomicAdd(&w[6], 1u);
                }
            }
            __syncthreads();
        }
        if (n > 1 && depth < SAH_DEPTH && threadIdx.x < 96) {
            const int ax = (int)(threadIdx.x >> 5);
            float c;
            int sp;
            sah_sweep_warp(s_bins[ax], c, sp);
            if ((threadIdx.x & 31u) == 0) {
                s_axc[ax] = ext[ax] > 0.0f ? c : INFINITY;
                s_axs[ax] = sp;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            int axis = -1, split = -1, leaf = 0;
            if (n <= 1) {
                leaf = 1;
            } else {
                float best_cost = INFINITY;
                if (depth < SAH_DEPTH) {
                    for (int ax = 0; ax < 3; ++ax)
                        if (s_axc[ax] < best_cost) { best_cost = s_axc[ax]; axis = ax; split = s_axs[ax]; }
                }
                const float parent_area = harea(v, v + 3);
                const float leaf_cost = (float)n;
                const float split_cost =
                    axis >= 0 ? trav_cost + (parent_area > 0 ? best_cost / parent_area : (float)n) : INFINITY;
                if (n <= (uint32_t)max_leaf && !(split_cost < leaf_cost)) leaf = 1;
            }
            s_pick[0] = axis;
            s_pick[1] = split;
            s_pick[2] = leaf;
            s_cnt[0] = s_cnt[1] = 0;
        }
        __syncthreads();
        const int axis = s_pick[0], split = s_pick[1];
        if (s_pick[2]) {
            if (threadIdx.x == 0) {
                // ascending primitive ids
                for (uint32_t i = lb + 1; i < le; ++i) {
                    const uint16_t x = s_perm[i];
                    uint32_t j = i;
                    while (j > lb && s_id[s_perm[j - 1]] > s_id[x]) { s_perm[j] = s_perm[j - 1]; --j; }
                    s_perm[j] = x;
                }
                DNode d;
                for (int k = 0; k < 3; ++k) { d.lo[k] = v[k]; d.hi[k] = v[3 + k]; }
                d.left = d.right = -1;
                d.start = slot_off + T.b + lb;
                d.count = n;
                nodes[node] = d;
            }
            __syncthreads();
            continue;
        }
        uint32_t mid;
        if (axis >= 0) {
            for (uint32_t i = lb + threadIdx.x; i < le; i += blockDim.x) {
                const uint16_t j = s_perm[i];
                const bool left = bin_of(0.5f * (s_box[j][axis] + s_box[j][3 + axis]), clo[axis], scale[axis]) < split;
                const uint32_t r = atomicAdd(&s_cnt[left ? 0 : 1], 1u);
                s_tmp[left ? lb + r : le - 1 - r] = j;
            }
            __syncthreads();
            mid = lb + s_cnt[0];
        } else {
            // object median on the widest centroid axis by (centroid, id)
            const int ax = widest_axis(clo, chi);
            for (uint32_t i = lb + threadIdx.x; i < le; i += blockDim.x) {
                const uint16_t j = s_perm[i];
                const float cj = 0.5f * (s_box[j][ax] + s_box[j][3 + ax]);
                const uint32_t idj = s_id[j];
                uint32_t rank = 0;
                for (uint32_t q = lb; q < le; ++q) {
                    const uint16_t x = s_perm[q];
                    const float cx = 0.5f * (s_box[x][ax] + s_box[x][3 + ax]);
                    rank += (cx < cj || (cx == cj && s_id[x] < idj)) ? 1u : 0u;
                }
                s_tmp[lb + rank] = j;
            }
            __syncthreads();
            mid = lb + n / 2;
        }
        for (uint32_t i = lb + threadIdx.x; i < le; i += blockDim.x) s_perm[i] = s_tmp[i];
        if (threadIdx.x == 0) {
            const uint32_t l = atomicAdd(node_ctr, 2u);
            if (l + 2 > node_cap || sp + 2 + (int)s_list_n > (int)SMALL) {
                atomicAdd(err, 1u);
                s_fail = 1;
            } else {
                DNode d;
                for (int k = 0; k < 3; ++k) { d.lo[k] = v[k]; d.hi[k] = v[3 + k]; }
                d.left = (int32_t)l;
                d.right = (int32_t)(l + 1);
                d.start = d.count = 0;
                nodes[node] = d;
                // right child first, so the left one is taken next
                const uint32_t cb[2] = {mid, lb}, ce[2] = {le, mid};
                int pushed = 0;
                for (int h = 0; h < 2; ++h) {
                    const uint32_t at = ce[h] - cb[h] <= WARP_SUBTREE ? SMALL - 1 - s_list_n++ : (uint32_t)(sp + pushed++);
                    s_stack[at] = make_uint2(l + 1 - h, cb[h] | (ce[h] << 16));
                    s_depth[at] = (uint16_t)(depth + 1);
                }
                s_push = pushed;
            }
        }
        __syncthreads();
        if (s_fail) break;
        sp += s_push;
    }
    __syncthreads();
    // phase 2: the subtrees of at most 32 primitives, one warp each
    if (!s_fail) {
        const uint32_t warp = threadIdx.x >> 5, lane = threadIdx.x & 31u;
        for (;;) {
            uint32_t item = 0;
            if (lane == 0) item = atomicAdd(&s_list_next, 1u);
            item = __shfl_sync(0xffffffffu, item, 0);
            if (item >= s_list_n) break;
            const uint32_t li = SMALL - 1 - item;
            if (!warp_subtree(s_stack[li], s_depth[li], s_box, s_id, s_perm, s_wstack[warp], s_wdepth[warp],
                              s_wbins[warp], nodes, node_ctr, node_cap,
                              slot_off + T.b, max_leaf, trav_cost)) {
                if (lane == 0) atomicAdd(err, 1u);
                break;
            }
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < n0; i += blockDim.x) idx[T.b + i] = s_id[s_perm[i]];
}

// ---------------------------------------------------- collapse + layout ---

__device__ __forceinline__ bool is_leaf(const DNode& d) { return d.left < 0; }

// One level of 4-wide nodes: each takes its binary node's children and
// keeps replacing the inner child of largest surface area by that child's
// two children until it has four (bvh_build.cpp children4); its inner
// children become the next level.
__global__ void k_collapse(const uint32_t* __restrict__ level, uint32_t nlevel, W4* __restrict__ w4,
                           uint32_t* __restrict__ w4_ctr, uint32_t* __restrict__ next, uint32_t* __restrict__ next_n,
                           const DNode* __restrict__ nodes) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nlevel) return;
    const uint32_t v = level[i];
    W4 w = w4[v];
    int32_t out[4] = {-1, -1, -1, -1};
    int n = 0;
    const DNode s = nodes[w.src];
    if (s.left >= 0) out[n++] = s.left;
    if (s.right >= 0) out[n++] = s.right;
    while (n < 4) {
        int best = -1;
        float best_area = -1.0f;
        for (int k = 0; k < n; ++k) {
            const DNode c = nodes[out[k]];
            if (is_leaf(c)) continue;
            const float a = harea(c.lo, c.hi);
            if (a > best_area) { best_area = a; best = k; }
        }
        if (best < 0) break;
        const DNode e = nodes[out[best]];
        int32_t kids[2];
        int nk = 0;
        if (e.left >= 0) kids[nk++] = e.left;
        if (e.right >= 0) kids[nk++] = e.right;
        if (nk == 0) break;
        out[best] = kids[0];
        if (nk == 2) out[n++] = kids[1];
    }
    w.n = n;
    for (int k = 0; k < 4; ++k) {
        w.child[k] = out[k];
        w.c4[k] = -1;
        if (k < n && !is_leaf(nodes[out[k]])) {
            const uint32_t c = atomicAdd(w4_ctr, 1u);
            W4 cw{};
            cw.src = out[k];
            cw.depth = w.depth + 1;
            w4[c] = cw;
            w.c4[k] = (int32_t)c;
            next[atomicAdd(next_n, 1u)] = c;
        }
    }
    w4[v] = w;
}

// Number of 4-wide nodes in each subtree (levels bottom-up).
__global__ void k_sizes(const uint32_t* __restrict__ level, uint32_t nlevel, const W4* __restrict__ w4,
                        uint32_t* __restrict__ size) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nlevel) return;
    const uint32_t v = level[i];
    uint32_t s = 1;
    for (int k = 0; k < 4; ++k)
        if (w4[v].c4[k] >= 0) s += size[w4[v].c4[k]];
    size[v] = s;
}

// Positions of the breadth-first top levels and the bases of the
// depth-first subtrees below them, in the host builder's queue order.
__global__ void k_layout_top(const W4* __restrict__ w4, const uint32_t* __restrict__ size, int bfs_levels,
                             uint32_t* __restrict__ pos, uint32_t* __restrict__ queue, uint32_t* __restrict__ frontier) {
    uint32_t qn = 0, qi = 0, fn = 0, next = 0;
    queue[qn++] = 0;
    while (qi < qn) {
        const uint32_t v = queue[qi++];
        if (w4[v].depth < bfs_levels) {
            pos[v] = next++;
            for (int k = 0; k < w4[v].n; ++k)
                if (w4[v].c4[k] >= 0) queue[qn++] = (uint32_t)w4[v].c4[k];
        } else {
            frontier[fn++] = v;
        }
    }
    for (uint32_t f = 0; f < fn; ++f) {
        pos[frontier[f]] = next;
        next += size[frontier[f]];
    }
}

// Depth-first positions below the breadth-first levels (levels top-down):
// children follow their parent in child order, each after the previous
// child's subtree.
__global__ void k_layout_down(const uint32_t* __restrict__ level, uint32_t nlevel, const W4* __restrict__ w4,
                              const uint32_t* __restrict__ size, uint32_t* __restrict__ pos) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nlevel) return;
    const uint32_t v = level[i];
    uint32_t run = pos[v] + 1;
    for (int k = 0; k < 4; ++k) {
        const int32_t c = w4[v].c4[k];
        if (c < 0) continue;
        pos[c] = run;
        run += size[c];
    }
}

struct Stats {
    unsigned long long leaves;
    double sah;
    uint32_t max_depth;
};

__global__ void k_write_nodes(const W4* __restrict__ w4, uint32_t n4, const uint32_t* __restrict__ pos,
                              const DNode* __restrict__ nodes, float* __restrict__ out, float root_area,
                              float trav_cost, Stats* __restrict__ st) {
    const uint32_t v = blockIdx.x * blockDim.x + threadIdx.x;
    if (v >= n4) return;
    const W4 w = w4[v];
    float* o = out + (size_t)pos[v] * (4 * BVH_NODE_F4);
    uint32_t leaves = 0;
    double sah = 0.0;
    for (int k = 0; k < 4; ++k) {
        int32_t ref = BVH_EMPTY;
        float lo[3] = {INFINITY, INFINITY, INFINITY}, hi[3] = {-INFINITY, -INFINITY, -INFINITY};
        if (k < w.n) {
            const DNode c = nodes[w.child[k]];
            for (int a = 0; a < 3; ++a) { lo[a] = c.lo[a]; hi[a] = c.hi[a]; }
            if (is_leaf(c)) {
                ref = ~(int32_t)((c.start << 3) | (c.count - 1));
                ++leaves;
                if (root_area > 0) sah += (double)(harea(c.lo, c.hi) / root_area * (float)c.count);
            } else {
                ref = (int32_t)pos[w.c4[k]];
            }
        }
        o[0 + k] = lo[0];
        o[4 + k] = hi[0];
        o[8 + k] = lo[1];
        o[12 + k] = hi[1];
        o[16 + k] = lo[2];
        o[20 + k] = hi[2];
        o[24 + k] = __int_as_float(ref);
        o[28 + k] = 0.0f;
    }
    const DNode s = nodes[w.src];
    if (root_area > 0) sah += (double)(trav_cost * harea(s.lo, s.hi) / root_area);
    atomicAdd(&st->leaves, (unsigned long long)leaves);
    atomicAdd(&st->sah, sah);
    atomicMax(&st->max_depth, (uint32_t)w.depth + 1);
}

// Device scratch released on every exit path.
struct Scratch {
    std::vector<void*> ptrs;
    ~Scratch() {
        for (void* p : ptrs) cudaFree(p);
    }
    template <typename T>
    T* get(size_t count, cudaError_t& e) {
        void* p = nullptr;
        if (e != cudaSuccess) return nullptr;
        e = dev_alloc(&p, std::max<size_t>(count, 1) * sizeof(T));
        if (e != cudaSuccess) return nullptr;
        ptrs.push_back(p);
        return static_cast<T*>(p);
    }
};

inline uint32_t blocks_for(uint64_t n, uint32_t t) { return (uint32_t)std::max<uint64_t>(1, (n + t - 1) / t); }

}  // namespace

bool build_bvh_device(const std::vector<PrimBox>* boxes, int ntypes, const uint32_t* slot_offset,
                      const BvhBuildParams& p, std::vector<uint32_t>* perm, FlatBvh& out, float4** d_nodes,
                      uint32_t* n_nodes, cudaStream_t st, std::string& err) {
    *d_nodes = nullptr;
    *n_nodes = 0;
    out = FlatBvh();
    size_t total = 0;
    for (int t = 0; t < ntypes; ++t) total += boxes[t].size();
    const int max_leaf = std::min(p.max_leaf, BVH_MAX_LEAF);
    cudaError_t e = cudaSuccess;
    auto fail = [&](const char* what) {
        err = std::string("device BVH build: ") + what + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
        return false;
    };
    if (total == 0) {
        // empty scene: the host builder's single node of empty children
        build_bvh(boxes, ntypes, slot_offset, p, perm, out);
        float4* dn = nullptr;
        if ((e = dev_alloc(&dn, out.nodes.size() * sizeof(float))) != cudaSuccess) return fail("cudaMalloc");
        e = cudaMemcpy(dn, out.nodes.data(), out.nodes.size() * sizeof(float), cudaMemcpyHostToDevice);
        if (e != cudaSuccess) { cudaFree(dn); return fail("cudaMemcpy"); }
        *d_nodes = dn;
        *n_nodes = (uint32_t)(out.nodes.size() / (4 * BVH_NODE_F4));
        return true;
    }
    Scratch S;
    const uint32_t node_cap = (uint32_t)(2 * total + 8);
    static_assert(sizeof(PrimBox) == 6 * sizeof(float), "PrimBox is six floats");
    float2* pb = S.get<float2>(3 * total, e);
    uint32_t* idx = S.get<uint32_t>(total, e);
    uint32_t* tmp = S.get<uint32_t>(total, e);
    DNode* nodes = S.get<DNode>(node_cap, e);
    uint32_t* ctr = S.get<uint32_t>(16, e);  // [0] nodes, [1] errors, [2] w4, [3] next level, [4..16) bounds
    if (e != cudaSuccess) return fail("cudaMalloc");
    {
        size_t o = 0;
        for (int t = 0; t < ntypes; ++t) {
            if (boxes[t].empty()) continue;
            e = cudaMemcpyAsync(pb + 3 * o, boxes[t].data(), boxes[t].size() * sizeof(PrimBox), cudaMemcpyHostToDevice, st);
            if (e != cudaSuccess) return fail("upload");
            o += boxes[t].size();
        }
    }
    // per-level buffers of the large-node phase, sized for the largest type:
    // its large nodes are disjoint and hold more than SMALL primitives each
    size_t max_n = 0;
    for (int t = 0; t < ntypes; ++t) max_n = std::max(max_n, boxes[t].size());
    const size_t lt_cap = max_n / (SMALL + 1) + 1, lc_cap = max_n / CHUNK + lt_cap + 1;
    LTask* dt = S.get<LTask>(lt_cap, e);
    LChunk* dc = S.get<LChunk>(lc_cap, e);
    uint32_t* bins = S.get<uint32_t>(lt_cap * LB_WORDS, e);
    uint32_t* ccnt = S.get<uint32_t>(lc_cap * 3 * NB, e);
    uint32_t* coff = S.get<uint32_t>(lc_cap * 2, e);
    LResult* dr = S.get<LResult>(lt_cap, e);
    if (e != cudaSuccess) return fail("cudaMalloc");
    if ((e = cudaMemsetAsync(ctr, 0, 16 * sizeof(uint32_t), st)) != cudaSuccess) return fail("memset");
    uint32_t host_nodes = 0;  // nodes allocated so far (the device counter after each sync)
    auto read_ctr = [&](uint32_t i, uint32_t& v) {
        e = cudaMemcpyAsync(&v, ctr + i, 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        return e == cudaSuccess;
    };
    auto set_ctr = [&](uint32_t i, uint32_t v) {
        e = cudaMemcpyAsync(ctr + i, &v, 4, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        return e == cudaSuccess;
    };
    auto put_node = [&](uint32_t i, const DNode& d) {
        e = cudaMemcpyAsync(nodes + i, &d, sizeof(DNode), cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        return e == cudaSuccess;
    };

    std::vector<int32_t> roots;
    std::vector<DNode> root_box;
    size_t type_base = 0;
    for (int t = 0; t < ntypes; ++t) {
        const uint32_t n = (uint32_t)boxes[t].size();
        perm[t].clear();
        if (n == 0) continue;
        const float2* tpb = pb + 3 * type_base;
        uint32_t* tidx = idx + type_base;
        uint32_t* ttmp = tmp + type_base;
        k_iota<<<blocks_for(n, 256), 256, 0, st>>>(tidx, n);
        // root bounds
        {
            uint32_t init[12];
            for (int k = 0; k < 12; ++k) init[k] = ((k % 6) < 3) ? 0xff800000u : 0x007fffffu;
            if ((e = cudaMemcpyAsync(ctr + 4, init, sizeof init, cudaMemcpyHostToDevice, st)) != cudaSuccess)
                return fail("memcpy");
            k_root_bounds<<<std::min<uint32_t>(blocks_for(n, 256), 1184), 256, 0, st>>>(tpb, n, ctr + 4);
        }
        uint32_t rb[12];
        if ((e = cudaMemcpyAsync(rb, ctr + 4, sizeof rb, cudaMemcpyDeviceToHost, st)) != cudaSuccess) return fail("memcpy");
        if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail("root bounds");
        float rv[12];
        for (int k = 0; k < 12; ++k) {
            const uint32_t u = rb[k];
            const uint32_t b = (u & 0x80000000u) ? (u & 0x7fffffffu) : ~u;
            std::memcpy(&rv[k], &b, 4);
        }
        if (!read_ctr(0, host_nodes)) return fail("counter");
        const uint32_t root = host_nodes++;
        if (!set_ctr(0, host_nodes)) return fail("counter");
        DNode rd;
        for (int k = 0; k < 3; ++k) { rd.lo[k] = rv[k]; rd.hi[k] = rv[3 + k]; }
        rd.left = rd.right = -1;
        rd.start = rd.count = 0;
        if (!put_node(root, rd)) return fail("node");
        roots.push_back((int32_t)root);
        root_box.push_back(rd);

        std::vector<LTask> large;
        std::vector<STask> small;
        if (n > SMALL) {
            LTask r{};
            r.node = root; r.b = 0; r.e = n; r.depth = 0;
            for (int k = 0; k < 3; ++k) { r.clo[k] = rv[6 + k]; r.chi[k] = rv[9 + k]; }
            large.push_back(r);
        } else {
            small.push_back(STask{root, 0, n, 0});
        }
        while (!large.empty()) {
            std::vector<LChunk> chunks;
            for (uint32_t i = 0; i < (uint32_t)large.size(); ++i) {
                LTask& T = large[i];
                T.chunk0 = (uint32_t)chunks.size();
                for (uint32_t b = T.b; b < T.e; b += CHUNK) chunks.push_back(LChunk{i, b, std::min(T.e, b + CHUNK)});
                T.nchunk = (uint32_t)chunks.size() - T.chunk0;
            }
            const uint32_t nt = (uint32_t)large.size(), nc = (uint32_t)chunks.size();
            if (nt > lt_cap || nc > lc_cap) return fail("level buffers");
            if ((e = cudaMemcpyAsync(dt, large.data(), nt * sizeof(LTask), cudaMemcpyHostToDevice, st)) != cudaSuccess ||
                (e = cudaMemcpyAsync(dc, chunks.data(), nc * sizeof(LChunk), cudaMemcpyHostToDevice, st)) != cudaSuccess)
                return fail("upload");
            k_init_bins<<<blocks_for((uint64_t)nt * LB_WORDS, 256), 256, 0, st>>>(bins, nt * LB_WORDS);
            k_bin_large<<<nc, 256, 0, st>>>(dt, dc, tidx, tpb, bins, ccnt);
            k_split_large<<<blocks_for(nt, 64), 64, 0, st>>>(dt, nt, bins, ccnt, nodes, ctr, node_cap, dr, coff, ctr + 1);
            k_partition_large<<<nc, 256, 0, st>>>(dt, dc, dr, coff, tidx, tpb, ttmp);
            k_copy_range<<<nc, 256, 0, st>>>(dc, dr, ttmp, tidx);
            std::vector<LResult> res(nt);
            if ((e = cudaMemcpyAsync(res.data(), dr, nt * sizeof(LResult), cudaMemcpyDeviceToHost, st)) != cudaSuccess)
                return fail("download");
            uint32_t errs = 0;
            if (!read_ctr(1, errs)) return fail("large split");
            if (errs) return fail("node capacity");
            if (!read_ctr(0, host_nodes)) return fail("counter");
            std::vector<LTask> next;
            for (uint32_t i = 0; i < nt; ++i) {
                const LTask& T = large[i];
                const LResult& R = res[i];
                uint32_t l, mid;
                float cl[2][3], ch[2][3];
                if (R.axis >= 0) {
                    l = R.left;
                    mid = R.mid;
                    std::memcpy(cl, R.clo, sizeof cl);
                    std::memcpy(ch, R.chi, sizeof ch);
                } else {
                    // object median by (centroid, id) on the host (no SAH split
                    // of a large node: all centroids equal, or depth >= 44)
                    std::vector<uint32_t> ids(T.e - T.b);
                    e = cudaMemcpyAsync(ids.data(), tidx + T.b, ids.size() * 4, cudaMemcpyDeviceToHost, st);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                    if (e != cudaSuccess) return fail("download");
                    const int ax = widest_axis(T.clo, T.chi);
                    const std::vector<PrimBox>& bx = boxes[t];
                    auto cen = [&](uint32_t x) { return 0.5f * (bx[x].lo[ax] + bx[x].hi[ax]); };
                    const size_t half = ids.size() / 2;
                    std::nth_element(ids.begin(), ids.begin() + half, ids.end(), [&](uint32_t x, uint32_t y) {
                        const float cx = cen(x), cy = cen(y);
                        return cx < cy || (cx == cy && x < y);
                    });
                    mid = T.b + (uint32_t)half;
                    l = host_nodes;
                    host_nodes += 2;
                    if (host_nodes > node_cap) return fail("node capacity");
                    if (!set_ctr(0, host_nodes)) return fail("counter");
                    DNode c[2];
                    for (int h = 0; h < 2; ++h) {
                        for (int k = 0; k < 3; ++k) {
                            c[h].lo[k] = cl[h][k] = INFINITY;
                            c[h].hi[k] = ch[h][k] = -INFINITY;
                        }
                        c[h].left = c[h].right = -1;
                        c[h].start = c[h].count = 0;
                        const size_t b0 = h ? half : 0, b1 = h ? ids.size() : half;
                        for (size_t q = b0; q < b1; ++q) {
                            const PrimBox& pbx = bx[ids[q]];
                            for (int k = 0; k < 3; ++k) {
                                const float cc = 0.5f * (pbx.lo[k] + pbx.hi[k]);
                                c[h].lo[k] = std::min(c[h].lo[k], pbx.lo[k]);
                                c[h].hi[k] = std::max(c[h].hi[k], pbx.hi[k]);
                                cl[h][k] = std::min(cl[h][k], cc);
                                ch[h][k] = std::max(ch[h][k], cc);
                            }
                        }
                        if (!put_node(l + h, c[h])) return fail("node");
                    }
                    DNode pn;
                    if ((e = cudaMemcpyAsync(&pn, nodes + T.node, sizeof pn, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
                        (e = cudaStreamSynchronize(st)) != cudaSuccess)
                        return fail("download");
                    pn.left = (int32_t)l;
                    pn.right = (int32_t)(l + 1);
                    if (!put_node(T.node, pn)) return fail("node");
                    e = cudaMemcpyAsync(tidx + T.b, ids.data(), ids.size() * 4, cudaMemcpyHostToDevice, st);
                    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
                    if (e != cudaSuccess) return fail("upload");
                }
                const uint32_t rng[2][2] = {{T.b, mid}, {mid, T.e}};
                for (int h = 0; h < 2; ++h) {
                    const uint32_t b = rng[h][0], en = rng[h][1];
                    if (en - b > SMALL) {
                        LTask c{};
                        c.node = l + h; c.b = b; c.e = en; c.depth = T.depth + 1;
                        for (int k = 0; k < 3; ++k) { c.clo[k] = cl[h][k]; c.chi[k] = ch[h][k]; }
                        next.push_back(c);
                    } else {
                        small.push_back(STask{l + (uint32_t)h, b, en, T.depth + 1});
                    }
                }
            }
            if ((e = cudaStreamSynchronize(st)) != cudaSuccess) return fail("large level");
            large.swap(next);
        }
        if (!small.empty()) {
            Scratch L;
            STask* ds = L.get<STask>(small.size(), e);
            if (e != cudaSuccess) return fail("cudaMalloc");
            if ((e = cudaMemcpyAsync(ds, small.data(), small.size() * sizeof(STask), cudaMemcpyHostToDevice, st)) !=
                cudaSuccess)
                return fail("upload");
            k_build_small<<<(uint32_t)small.size(), SB_THREADS, 0, st>>>(ds, tidx, tpb, nodes, ctr, node_cap,
                                                                          slot_offset[t], max_leaf, p.trav_cost, ctr + 1);
            if ((e = cudaGetLastError()) != cudaSuccess) return fail("small subtrees");
            uint32_t errs = 0;
            if (!read_ctr(1, errs)) return fail("small subtrees");
            if (errs) return fail("node capacity");
            if (!read_ctr(0, host_nodes)) return fail("counter");
        }
        perm[t].resize(n);
        e = cudaMemcpyAsync(perm[t].data(), tidx, (size_t)n * 4, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        if (e != cudaSuccess) return fail("download");
        type_base += n;
    }

    // join the type roots pairwise (bvh_build.cpp), wrap a single leaf
    while (roots.size() > 1) {
        DNode j;
        const DNode& a = root_box[root_box.size() - 2];
        const DNode& b = root_box[root_box.size() - 1];
        for (int k = 0; k < 3; ++k) { j.lo[k] = std::min(a.lo[k], b.lo[k]); j.hi[k] = std::max(a.hi[k], b.hi[k]); }
        j.left = roots[roots.size() - 2];
        j.right = roots[roots.size() - 1];
        j.start = j.count = 0;
        const uint32_t id = host_nodes++;
        if (!put_node(id, j)) return fail("node");
        roots.pop_back();
        root_box.pop_back();
        roots.back() = (int32_t)id;
        root_box.back() = j;
    }
    int32_t root = roots[0];
    {
        DNode r;
        if ((e = cudaMemcpyAsync(&r, nodes + root, sizeof r, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return fail("download");
        if (r.left < 0) {
            DNode wr = r;
            wr.left = root;
            wr.right = -1;
            wr.start = wr.count = 0;
            root = (int32_t)host_nodes++;
            if (!put_node((uint32_t)root, wr)) return fail("node");
        }
        root_box.back() = r;
    }
    const float root_area = harea(root_box.back().lo, root_box.back().hi);

    // collapse level by level
    const uint32_t w4_cap = host_nodes;
    W4* w4 = S.get<W4>(w4_cap, e);
    uint32_t* lvl = S.get<uint32_t>(w4_cap, e);
    uint32_t* size = S.get<uint32_t>(w4_cap, e);
    uint32_t* pos = S.get<uint32_t>(w4_cap, e);
    uint32_t* queue = S.get<uint32_t>(w4_cap, e);
    uint32_t* frontier = S.get<uint32_t>(w4_cap, e);
    Stats* dstat = S.get<Stats>(1, e);
    if (e != cudaSuccess) return fail("cudaMalloc");
    {
        W4 r{};
        r.src = root;
        uint32_t zero = 0, one = 1;
        if ((e = cudaMemcpyAsync(w4, &r, sizeof r, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemcpyAsync(lvl, &zero, 4, cudaMemcpyHostToDevice, st)) != cudaSuccess ||
            (e = cudaMemsetAsync(dstat, 0, sizeof(Stats), st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return fail("upload");
        if (!set_ctr(2, one)) return fail("counter");
    }
    std::vector<uint32_t> lvl_off{0, 1};
    for (;;) {
        const uint32_t b = lvl_off[lvl_off.size() - 2], en = lvl_off.back(), cnt = en - b;
        if (cnt == 0) break;
        if (!set_ctr(3, 0)) return fail("counter");
        k_collapse<<<blocks_for(cnt, 128), 128, 0, st>>>(lvl + b, cnt, w4, ctr + 2, lvl + en, ctr + 3, nodes);
        uint32_t nn = 0;
        if (!read_ctr(3, nn)) return fail("collapse");
        lvl_off.push_back(en + nn);
    }
    const uint32_t n4 = lvl_off.back();
    const int nlev = (int)lvl_off.size() - 2;  // levels 0..nlev-1 are non-empty
    for (int l = nlev - 1; l >= 0; --l) {
        const uint32_t b = lvl_off[l], cnt = lvl_off[l + 1] - b;
        k_sizes<<<blocks_for(cnt, 128), 128, 0, st>>>(lvl + b, cnt, w4, size);
    }
    const int bfs = std::max(0, p.top_bfs_levels);
    k_layout_top<<<1, 1, 0, st>>>(w4, size, bfs, pos, queue, frontier);
    for (int l = bfs; l < nlev; ++l) {
        const uint32_t b = lvl_off[l], cnt = lvl_off[l + 1] - b;
        k_layout_down<<<blocks_for(cnt, 128), 128, 0, st>>>(lvl + b, cnt, w4, size, pos);
    }
    float* dn = nullptr;
    if ((e = dev_alloc(&dn, (size_t)n4 * BVH_NODE_BYTES)) != cudaSuccess) return fail("cudaMalloc");
    k_write_nodes<<<blocks_for(n4, 128), 128, 0, st>>>(w4, n4, pos, nodes, dn, root_area, p.trav_cost, dstat);
    Stats hs{};
    out.nodes.assign(4 * BVH_NODE_F4, 0.0f);
    if ((e = cudaGetLastError()) != cudaSuccess ||
        (e = cudaMemcpyAsync(&hs, dstat, sizeof hs, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaMemcpyAsync(out.nodes.data(), dn, BVH_NODE_BYTES, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess) {
        cudaFree(dn);
        return fail("layout");
    }
    out.stats.inner_nodes = n4;
    out.stats.leaves = (uint32_t)hs.leaves;
    out.stats.max_depth = hs.max_depth;
    out.stats.sah_cost = hs.sah;
    *d_nodes = reinterpret_cast<float4*>(dn);
    *n_nodes = n4;
    return true;
}

}  // namespace cupbr_b200

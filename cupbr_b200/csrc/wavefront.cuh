// Device building blocks shared by the wavefront renderers (path tracer and
// density-grid medium): warp-aggregated queue slots and the persistent
// traversal loop over a ray queue.
#pragma once

#include "dev_common.cuh"
#include "trace.cuh"

namespace cupbr_b200 {

__device__ __forceinline__ uint32_t lane_id() { return threadIdx.x & 31u; }

// Loads of wavefront state (queues, hits, radiance, counters).  NC = true:
// the read-only path (__ldg), for stage kernels, which never read what they
// themselves write.  NC = false: cached in L2 only (__ldcg), for the
// persistent batch kernel, whose stages read what other blocks of the same
// launch wrote before a grid barrier (an L1 or read-only cache line from an
// earlier stage could be stale).
template <bool NC, typename T>
__device__ __forceinline__ T qload(const T* p) {
    return NC ? __ldg(p) : __ldcg(p);
}

// Warp-aggregated slot allocation for the lanes with `want` set.
__device__ __forceinline__ uint32_t claim_slot(bool want, uint32_t* counter) {
    const unsigned full = 0xffffffffu;
    unsigned mask = __ballot_sync(full, want);
    if (mask == 0u) return 0u;
    int leader = __ffs(mask) - 1;
    uint32_t base = 0;
    if ((int)lane_id() == leader) base = atomicAdd(counter, (uint32_t)__popc(mask));
    base = __shfl_sync(full, base, leader);
    return base + (uint32_t)__popc(mask & ((1u << lane_id()) - 1u));
}

// Persistent traversal over a queue with per-lane dynamic fetch: lanes whose
// ray finished take the next rays of the queue (one atomicAdd per warp for
// all of them) while the others resume their traversal, so a warp stays full
// until the queue runs dry.  Entry i of the queue starts at q[stride * i]:
// (origin, ANY ? t_limit : -), (direction, -).  ANY = false: closest hit,
// ANY = true: occlusion up to t_limit.  done(i, state) runs once per ray.
// The top smem_nodes BVH nodes are staged in shared memory (s_nodes).
template <bool ANY, bool COUNT, bool NC = true, typename Done>
__device__ __forceinline__ void persistent_trace(const DeviceScene& S, const float4* __restrict__ q, uint32_t stride,
                                                 uint32_t count, uint32_t* fetch, uint32_t smem_nodes,
                                                 float4* s_nodes, uint32_t* err_stack, uint64_t* stats, Done done) {
    // a block that starts after the queue has been handed out (or on an empty
    // queue) leaves before staging the top of the tree; the decision is the
    // block's (the counter can move between two threads' reads)
    if (!__syncthreads_or(*(volatile const uint32_t*)fetch < count)) return;
    const uint32_t nsm = min(S.n_nodes, smem_nodes);
    for (uint32_t i = threadIdx.x; i < nsm * BVH_NODE_F4; i += blockDim.x) s_nodes[i] = __ldg(&S.nodes[i]);
    __syncthreads();

    const unsigned full = 0xffffffffu;
    const uint32_t lane = lane_id();
    TravState s;
    int32_t st_ref[CUPBR_STACK_SIZE];
    float st_t[CUPBR_STACK_SIZE];
    TraceCounters tc;
    bool overflow = false, have = false, exhausted = false;
    uint32_t idx = 0;
    for (;;) {
        const bool want = !have && !exhausted;
        const unsigned m = __ballot_sync(full, want);
        if (m) {
            const int leader = __ffs(m) - 1;
            uint32_t base = 0;
            if ((int)lane == leader) base = atomicAdd(fetch, (uint32_t)__popc(m));
            base = __shfl_sync(full, base, leader);
            if (want) {
                idx = base + (uint32_t)__popc(m & ((1u << lane) - 1u));
                if (idx < count) {
                    const float4 q0 = qload<NC>(&q[stride * (size_t)idx]);
                    const float4 q1 = qload<NC>(&q[stride * (size_t)idx + 1]);
                    trav_init<ANY>(S, s, xyz(q0), xyz(q1), ANY ? q0.w : 0.0f);
                    have = true;
                } else {
                    exhausted = true;
                }
            }
        }
        if (!__ballot_sync(full, have)) break;
        if (have) {
            // two descent + leaf rounds between refills (measured best: one round
            // pays the refill too often, four or more let finished lanes idle)
            trav_run<ANY, COUNT>(S, s_nodes, nsm, s, st_ref, st_t, 2, overflow, tc);
            if (s.done) {
                have = false;
                done(idx, s);
            }
        }
    }
    if (overflow) atomicAdd(err_stack, 1u);
    if (COUNT) {
        atomicAdd((unsigned long long*)&stats[0], (unsigned long long)tc.nodes);
        atomicAdd((unsigned long long*)&stats[1], (unsigned long long)tc.tris);
    }
}

// Queue slot of a frame -> pixel.  Slots go by 32 over 8x4 pixel tiles
// (tiles row by row), so the camera rays a traversal warp fetches together
// cover a compact patch of the screen and walk nearly the same nodes; the
// right and bottom strips the tiles leave (width % 8, height % 4) follow
// row by row.  A bijection on [0, w * h).
__device__ __forceinline__ uint32_t slot_pixel(uint32_t s, uint32_t w, uint32_t h) {
    const uint32_t tx = w >> 3, h4 = h & ~3u;
    const uint32_t tiled = tx * 8u * h4;
    if (s < tiled) {
        const uint32_t t = s >> 5, l = s & 31u;
        const uint32_t ty = t / tx, tt = t - ty * tx;
        return (ty * 4u + (l >> 3)) * w + tt * 8u + (l & 7u);
    }
    s -= tiled;
    const uint32_t rw = w - tx * 8u;
    if (s < rw * h4) {
        const uint32_t y = s / rw;
        return y * w + tx * 8u + (s - y * rw);
    }
    return h4 * w + (s - rw * h4);
}

// Closest hits of one warp's 32 rays walked as a packet (packet_visit4):
// every lane of the warp calls it together; a lane with valid = false takes
// part in the walk but accepts no box.  On return s holds the lane's hit as
// trav_run leaves it (t_best, best_prim, best_key).
__device__ __forceinline__ void packet_closest(const DeviceScene& S, const float4* s_nodes, uint32_t nsm, f3 o, f3 d,
                                               bool valid, TravState& s, int32_t* st_ref, float* st_t,
                                               bool& overflow) {
    trav_init<false>(S, s, o, d, 0.0f);
    // a lane past the end of the queue accepts no box (t_f <= -1 < t_n)
    if (!valid) s.t_best = -1.0f;
    int sp = 0;
    int32_t cur = 0;
    uint32_t guard = 2u * S.n_nodes + 64u;
    bool live = S.n_nodes != 0;
    while (live) {
        if (cur >= 0) {
            if (--guard == 0u || (uint32_t)cur >= S.n_nodes) { overflow = true; break; }
            float4 nb[7];
            fetch_node(S, s_nodes, nsm, cur, nb);
            int32_t first;
            if (packet_visit4(nb, s.idir, s.ood, s.t_best, first, st_ref, st_t, sp, overflow)) cur = first;
            else live = packet_pop(s.t_best, st_ref, st_t, sp, cur);
        } else {
            if (valid) trav_leaf_closest(S, s, ~(uint32_t)cur);
            live = packet_pop(s.t_best, st_ref, st_t, sp, cur);
        }
    }
}

// Closest hits of a coherent queue as warp packets (packet_visit4): each
// warp takes 32 consecutive entries, which the camera kernel fills from
// one 8x4 pixel tile, and walks the tree once for all of them.  The
// entries, their hits and done(i, state) are those of persistent_trace;
// only the traversal order differs, which the closest hit does not depend
// on.  No traversal counters (instrumented frames use persistent_trace).
template <bool NC = true, typename Done>
__device__ __forceinline__ void packet_trace(const DeviceScene& S, const float4* __restrict__ q, uint32_t stride,
                                             uint32_t count, uint32_t* fetch, uint32_t smem_nodes, float4* s_nodes,
                                             uint32_t* err_stack, Done done) {
    if (!__syncthreads_or(*(volatile const uint32_t*)fetch < count)) return;  // as persistent_trace
    const uint32_t nsm = min(S.n_nodes, smem_nodes);
    for (uint32_t i = threadIdx.x; i < nsm * BVH_NODE_F4; i += blockDim.x) s_nodes[i] = __ldg(&S.nodes[i]);
    __syncthreads();

    const unsigned full = 0xffffffffu;
    const uint32_t lane = lane_id();
    int32_t st_ref[CUPBR_STACK_SIZE];
    float st_t[CUPBR_STACK_SIZE];
    bool overflow = false;
    for (;;) {
        uint32_t base = 0;
        if (lane == 0) base = atomicAdd(fetch, 32u);
        base = __shfl_sync(full, base, 0);
        if (base >= count) break;
        const uint32_t idx = base + lane;
        const bool valid = idx < count;
        f3 o = mk(0.0f, 0.0f, 0.0f), d = mk(0.0f, 0.0f, 1.0f);
        if (valid) {
            o = xyz(qload<NC>(&q[stride * (size_t)idx]));
            d = xyz(qload<NC>(&q[stride * (size_t)idx + 1]));
        }
        TravState s;
        packet_closest(S, s_nodes, nsm, o, d, valid, s, st_ref, st_t, overflow);
        if (valid) done(idx, s);
    }
    if (overflow) atomicAdd(err_stack, 1u);
}

}  // namespace cupbr_b200

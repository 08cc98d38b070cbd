// trace_kernels.cu — closest-hit and any-hit wavefront kernels over the
// compressed BVH8 (the ray queries of shader.wgsl:561-566 and :654-659).
//
// Kept in their own translation unit: the traversal is compiled with
// multiply-add contraction (fast slab tests), while the shading kernels are
// compiled without it so that they round like the CPU oracle.
//
// Persistent warps with dynamic ray fetch (Aila and Laine, HPG 2009): the
// grid holds one wave of resident blocks; each warp draws queue positions
// from a counter, and once REFILL lanes have finished their rays the warp
// hands those lanes new rays, so divergent ray lengths do not idle lanes.
// The shared-memory stack is sized to the tree: STACK = 16 entries for trees
// of at most 16 levels (config 2 builds 10), 32 otherwise.
#include <algorithm>

#include "render_kernels.h"

// 8 resident blocks of 128 threads per SM caps the kernels at 64 registers:
// the unbounded build takes ~110 and halves the warps in flight (measured:
// 8.7 ms vs 6.1 ms of closest-hit traversal per config-2 frame).
#ifndef SRT_TRACE_MIN_BLOCKS
#define SRT_TRACE_MIN_BLOCKS 8
#endif
// resident blocks per SM the batch's persistent kernel (k_trace_multi_pt) is
// compiled for (its launch takes the batch's tuned blocks per SM, at most this)
#ifndef SRT_TRACE_MULTI_BLOCKS
#define SRT_TRACE_MULTI_BLOCKS SRT_TRACE_MIN_BLOCKS
#endif
// resident blocks of the persistent kernel (k_trace_pt) per SM: 9 caps it at
// 56 registers without spills of the closest-hit form (a 4-byte spill in the
// any-hit form); config-2 frame 9.16 vs 9.43 ms with 8 (closest-hit bounces
// 1-4 6 % faster, photon pass 2.45 vs 2.54 ms).  The one-ray-per-thread
// kernel stays at 8 (bounce 0 0.44 vs 0.42 ms with 9); 10 blocks (48
// registers) spill: 9.43 ms.
#ifndef SRT_TRACE_PT_BLOCKS
#define SRT_TRACE_PT_BLOCKS 9
#endif
// idle lanes that trigger a refill of the warp: closest-hit and any-hit
// kernels (config-2 frame, refill at 4 / 6 / 8 / 12 / 16 / 20 idle lanes for
// both: 10.01 / 9.96 / 9.94 / 9.97 / 10.10 / 10.31 ms; closest-hit traversal is
// fastest at 6, any-hit at 12)
#ifndef SRT_TRACE_REFILL
#define SRT_TRACE_REFILL 6
#endif
#ifndef SRT_TRACE_REFILL_ANY
#define SRT_TRACE_REFILL_ANY 12
#endif
#ifndef SRT_TRACE_PERSISTENT
#define SRT_TRACE_PERSISTENT 1
#endif
// first bounce whose shadow rays use persistent warps (> 31: none).  Shadow
// rays of bounces >= 1 are incoherent, and refilling idle lanes pays
// (config-2 shadow rays 2.38 vs 2.61 ms per frame); with the pooled triangle
// tests bounce 0's do too (0.41 vs 0.45 ms).
#ifndef SRT_SHADOW_PERSISTENT_FROM
#define SRT_SHADOW_PERSISTENT_FROM 0
#endif

// camera rays of bounce 0 in persistent warps (k_trace_pt) instead of one
// per thread: measured slower (0.44 vs 0.42 ms per config-2 frame), the
// pixel-ordered rays are coherent and end together
#ifndef SRT_PRIMARY_PERSISTENT
#define SRT_PRIMARY_PERSISTENT 0
#endif
// photon rays in persistent warps (k_trace_pt) instead of one per thread:
// with the warp-synchronous node visits the refill pays (photon pass 2.53 vs
// 2.62 ms per config-2 frame; before it, 3.35 vs 3.15)
#ifndef SRT_PHOTON_PERSISTENT
#define SRT_PHOTON_PERSISTENT 1
#endif

// Fetch the next node with cp.async into shared memory while the pending
// triangle tests run (k_trace and k_trace_pt).
#ifndef SRT_TRAV_PREFETCH
#define SRT_TRAV_PREFETCH 0
#endif

namespace srt {

namespace {

constexpr bool kPrefetch = SRT_TRAV_PREFETCH != 0;
constexpr bool kPool = SRT_TRAV_POOL != 0 && !kPrefetch;

// Dynamic shared memory of a traversal block: the stacks, then (prefetch)
// 5 x uint4 node slots per thread.
template <int STACK>
constexpr size_t trace_smem() {
    return sizeof(uint2) * STACK * TRACE_BLOCK + (kPrefetch ? sizeof(uint4) * 5 * TRACE_BLOCK : 0);
}
template <int STACK>
SRT_DEV uint4* node_slots(uint2* smem) {
    return reinterpret_cast<uint4*>(smem + STACK * TRACE_BLOCK) + threadIdx.x;
}

// One ray per thread, one launch over the whole queue.
template <bool ANY, bool COUNT, int STACK>
__global__ void __launch_bounds__(TRACE_BLOCK, SRT_TRACE_MIN_BLOCKS)
    k_trace(DevScene S, const uint32_t* __restrict__ queue, const uint32_t* __restrict__ count,
            const float4* __restrict__ ro, const float4* __restrict__ rd, float4* __restrict__ hit,
            const uint32_t* __restrict__ sh_id, const float4* __restrict__ sh_c, float4* __restrict__ rad,
            uint32_t* err, DevStats* stats, int kind, int bounce) {
    extern __shared__ uint2 stack_smem[];
    uint32_t q = blockIdx.x * TRACE_BLOCK + threadIdx.x;
    uint32_t n = *count;
    if (q >= n) return;
    uint32_t id = queue ? queue[q] : q;
    float4 o = ro[ANY ? q : id], d = rd[ANY ? q : id];
    Ray ray{xyz(o), xyz(d), o.w, d.w};
    float t = 0.f, u = 0.f, v = 0.f;
    uint32_t prim;
    TravCounters tc{&stats->nodes_bounce[kind][bounce], &stats->tris_bounce[kind][bounce]};
    bool h = traverse<ANY, COUNT, STACK, kPrefetch>(S, ray, stack_smem + threadIdx.x, TRACE_BLOCK, t, prim, u, v, err,
                                                    tc, kPrefetch ? node_slots<STACK>(stack_smem) : nullptr);
    if (ANY) {
        // shadow ray: unoccluded -> add its contribution (shader.wgsl:659-669)
        if (!h) {
            uint32_t pid = sh_id[q];
            float4 c = sh_c[q], r = rad[pid];
            rad[pid] = make_float4(__fadd_rn(r.x, c.x), __fadd_rn(r.y, c.y), __fadd_rn(r.z, c.z), __fadd_rn(r.w, c.w));
        }
    } else {
        hit[id] = h ? make_float4(t, __uint_as_float(prim), u, v) : make_float4(0.f, __uint_as_float(MISS), 0.f, 0.f);
    }
}

// Persistent form: same inputs and outputs, queue positions from *fetch.
template <bool ANY, bool COUNT, int STACK>
__global__ void __launch_bounds__(TRACE_BLOCK, SRT_TRACE_PT_BLOCKS)
    k_trace_pt(DevScene S, const uint32_t* __restrict__ queue, const uint32_t* __restrict__ count,
               uint32_t* __restrict__ fetch, const float4* __restrict__ ro, const float4* __restrict__ rd,
               float4* __restrict__ hit, const uint32_t* __restrict__ sh_id, const float4* __restrict__ sh_c,
               float4* __restrict__ rad, uint32_t* err, DevStats* stats, int kind, int bounce) {
    extern __shared__ uint2 stack_smem[];
    uint2* stack = stack_smem + threadIdx.x;
    const uint32_t n = *count;
    if (n == 0u) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt = (1u << lane) - 1u;
    TravState T;
    bool active = false, exhausted = false;
    uint32_t q = 0, id = 0, n_nodes = 0, n_tris = 0;
    while (true) {
        uint32_t idle = __ballot_sync(0xFFFFFFFFu, !active);
        if (!exhausted && __popc(idle) >= (ANY ? SRT_TRACE_REFILL_ANY : SRT_TRACE_REFILL)) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(fetch, (uint32_t)__popc(idle));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base + (uint32_t)__popc(idle) >= n) exhausted = true;
            if (!active) {
                uint32_t my = base + __popc(idle & lt);
                if (my < n) {
                    q = my;
                    id = queue ? queue[q] : q;
                    float4 o = ro[ANY ? q : id], d = rd[ANY ? q : id];
                    active = trav_init(T, S, xyz(o), xyz(d), o.w, d.w);
                    if (!active) {  // degenerate ray: finished without a hit
                        if (ANY) {
                            uint32_t pid = sh_id[q];
                            float4 c = sh_c[q], r = rad[pid];
                            rad[pid] = make_float4(__fadd_rn(r.x, c.x), __fadd_rn(r.y, c.y), __fadd_rn(r.z, c.z),
                                                   __fadd_rn(r.w, c.w));
                        } else {
                            hit[id] = make_float4(0.f, __uint_as_float(MISS), 0.f, 0.f);
                        }
                    }
                }
            }
        }
        if (__ballot_sync(0xFFFFFFFFu, active) == 0u) {
            if (exhausted) break;
            continue;
        }
        if (kPool && (ANY || SRT_TRAV_POOL >= 2)) {
            // the triangles of the lanes' last node visits, dealt out over the warp
            pool_tris<ANY>(S, T, active, n_tris);
            if (ANY && active && T.best != MISS) active = false;  // occluded: nothing to add
        }
        if (active && trav_step<ANY, STACK, kPrefetch>(S, T, stack, TRACE_BLOCK, err, n_nodes, n_tris,
                                                       kPrefetch ? node_slots<STACK>(stack_smem) : nullptr)) {
            active = false;
            if (ANY) {
                if (T.best == MISS) {
                    uint32_t pid = sh_id[q];
                    float4 c = sh_c[q], r = rad[pid];
                    rad[pid] = make_float4(__fadd_rn(r.x, c.x), __fadd_rn(r.y, c.y), __fadd_rn(r.z, c.z),
                                           __fadd_rn(r.w, c.w));
                }
            } else {
                hit[id] = T.best != MISS ? make_float4(T.tbest, __uint_as_float(T.best), T.bu, T.bv)
                                         : make_float4(0.f, __uint_as_float(MISS), 0.f, 0.f);
            }
        }
    }
    if (COUNT) {
        atomicAdd(&stats->nodes_bounce[kind][bounce], (unsigned long long)n_nodes);
        atomicAdd(&stats->tris_bounce[kind][bounce], (unsigned long long)n_tris);
    }
}

template <bool ANY>
__global__ void __launch_bounds__(TRACE_BLOCK) k_trace_batch(DevScene S, const float4* __restrict__ rays, uint32_t n,
                                                             float4* __restrict__ hits, uint32_t* err) {
    extern __shared__ uint2 stack_smem[];
    uint32_t i = blockIdx.x * TRACE_BLOCK + threadIdx.x;
    if (i >= n) return;
    float4 o = rays[2 * i], d = rays[2 * i + 1];
    Ray ray{xyz(o), xyz(d), o.w, d.w};
    float t = 0.f, u = 0.f, v = 0.f;
    uint32_t prim;
    TravCounters tc{nullptr, nullptr};
    bool h = traverse<ANY, false>(S, ray, stack_smem + threadIdx.x, TRACE_BLOCK, t, prim, u, v, err, tc);
    if (ANY) hits[i] = make_float4(h ? t : 0.f, __uint_as_float(h ? 0u : MISS), 0.f, 0.f);
    else hits[i] = h ? make_float4(t, __uint_as_float(prim), u, v) : make_float4(0.f, __uint_as_float(MISS), 0.f, 0.f);
}

// Rays of many scenes in one launch (the batched renderer): a virtual queue
// concatenates every item's rays, each item padded to whole chunks, so a
// warp's chunk never straddles two scenes; warps draw chunks from *fetch
// and trace them lane per ray (persistent, no refill).
template <bool ANY, int STACK>
__global__ void __launch_bounds__(TRACE_BLOCK, SRT_TRACE_MIN_BLOCKS)
    k_trace_multi(const MultiTraceItem* __restrict__ items, int n_items, uint32_t* __restrict__ fetch,
                  uint32_t chunk) {
    extern __shared__ uint2 stack_smem[];
    __shared__ uint32_t pre[MAX_BATCH + 1];
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int i = 0; i < n_items; ++i) {
            pre[i] = acc;
            acc += (*items[i].count + chunk - 1u) / chunk * chunk;
        }
        pre[n_items] = acc;
    }
    __syncthreads();
    const uint32_t total = pre[n_items];
    const uint32_t lane = threadIdx.x & 31u;
    uint2* stack = stack_smem + threadIdx.x;
    while (true) {
        uint32_t g = 0;
        if (lane == 0) g = atomicAdd(fetch, chunk);
        g = __shfl_sync(0xFFFFFFFFu, g, 0);
        if (g >= total) break;
        int s = 0;
        while (s + 1 < n_items && pre[s + 1] <= g) ++s;
        const MultiTraceItem& I = items[s];
        const uint32_t n = *I.count;
        for (uint32_t k = 0; k < chunk; k += 32u) {
            const uint32_t q = g - pre[s] + k + lane;
            if (q >= n) continue;
            const uint32_t id = I.queue ? I.queue[q] : q;
            float4 o = I.ro[ANY ? q : id], d = I.rd[ANY ? q : id];
            Ray ray{xyz(o), xyz(d), o.w, d.w};
            float t = 0.f, u = 0.f, v = 0.f;
            uint32_t prim;
            TravCounters tc{nullptr, nullptr};
            bool h = traverse<ANY, false, STACK>(I.s, ray, stack, TRACE_BLOCK, t, prim, u, v, I.err, tc);
            if (ANY) {
                if (!h) {
                    uint32_t pid = I.sh_id[q];
                    float4 c = I.sh_c[q], r = I.rad[pid];
                    I.rad[pid] = make_float4(__fadd_rn(r.x, c.x), __fadd_rn(r.y, c.y), __fadd_rn(r.z, c.z),
                                             __fadd_rn(r.w, c.w));
                }
            } else {
                I.hit[id] = h ? make_float4(t, __uint_as_float(prim), u, v)
                              : make_float4(0.f, __uint_as_float(MISS), 0.f, 0.f);
            }
        }
    }
}

// Persistent form of the batch's traversal (SRT_BATCH_TRACE_PT): the lanes
// of a warp take rays from one virtual queue over every item's rays (no
// padding) and keep their own scene, so a finished lane takes the next ray
// whatever scene it belongs to; the steps are those of k_trace_pt (closest
// hits with the warp-synchronous node visit, any-hit rays with pooled
// triangle tests that read the owner's scene).
template <bool ANY, int STACK>
__global__ void __launch_bounds__(TRACE_BLOCK, SRT_TRACE_MULTI_BLOCKS)
    k_trace_multi_pt(const MultiTraceItem* __restrict__ items, int n_items, uint32_t* __restrict__ fetch) {
    extern __shared__ uint2 stack_smem[];
    __shared__ uint32_t pre[MAX_BATCH + 1];
    if (threadIdx.x == 0) {
        uint32_t acc = 0;
        for (int i = 0; i < n_items; ++i) {
            pre[i] = acc;
            acc += *items[i].count;
        }
        pre[n_items] = acc;
    }
    __syncthreads();
    const uint32_t total = pre[n_items];
    if (total == 0u) return;
    const uint32_t lane = threadIdx.x & 31u;
    const uint32_t lt = (1u << lane) - 1u;
    uint2* stack = stack_smem + threadIdx.x;
    DevScene S;  // this lane's scene: the fields traversal reads
    S.nodes = nullptr;
    S.tris = nullptr;
    S.n_nodes = 0u;
    TravState T{};
    bool active = false, exhausted = false;
    uint32_t q = 0, id = 0, n_nodes = 0, n_tris = 0;
    int s = 0;
    // a finished ray: the closest hit, or an unoccluded shadow ray's contribution
    auto finish = [&](const MultiTraceItem& I) {
        if (ANY) {
            if (T.best == MISS) {
                const uint32_t pid = I.sh_id[q];
                const float4 c = I.sh_c[q], r = I.rad[pid];
                I.rad[pid] = make_float4(__fadd_rn(r.x, c.x), __fadd_rn(r.y, c.y), __fadd_rn(r.z, c.z),
                                         __fadd_rn(r.w, c.w));
            }
        } else {
            I.hit[id] = T.best != MISS ? make_float4(T.tbest, __uint_as_float(T.best), T.bu, T.bv)
                                       : make_float4(0.f, __uint_as_float(MISS), 0.f, 0.f);
        }
    };
    while (true) {
        const uint32_t idle = __ballot_sync(0xFFFFFFFFu, !active);
        if (!exhausted && __popc(idle) >= (ANY ? SRT_TRACE_REFILL_ANY : SRT_TRACE_REFILL)) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(fetch, (uint32_t)__popc(idle));
            base = __shfl_sync(0xFFFFFFFFu, base, 0);
            if (base + (uint32_t)__popc(idle) >= total) exhausted = true;
            if (!active) {
                const uint32_t my = base + __popc(idle & lt);
                if (my < total) {
                    // the item holding virtual index `my`: the last with pre[i] <= my
                    int lo = 0, hi = n_items - 1;
                    while (lo < hi) {
                        const int mid = (lo + hi + 1) >> 1;
                        if (pre[mid] <= my) lo = mid;
                        else hi = mid - 1;
                    }
                    s = lo;
                    const MultiTraceItem& I = items[s];
                    S.nodes = I.s.nodes;
                    S.tris = I.s.tris;
                    S.n_nodes = I.s.n_nodes;
                    q = my - pre[s];
                    id = I.queue ? I.queue[q] : q;
                    const float4 o = I.ro[ANY ? q : id], d = I.rd[ANY ? q : id];
                    active = trav_init(T, S, xyz(o), xyz(d), o.w, d.w);
                    if (!active) finish(I);  // degenerate ray: finished without a hit
                }
            }
        }
        if (__ballot_sync(0xFFFFFFFFu, active) == 0u) {
            if (exhausted) break;
            continue;
        }
        if (kPool && (ANY || SRT_TRAV_POOL >= 2)) {
            pool_tris<ANY, true>(S, T, active, n_tris);
            if (ANY && active && T.best != MISS) active = false;  // occluded: nothing to add
        }
        if (active && trav_step<ANY, STACK>(S, T, stack, TRACE_BLOCK, items[s].err, n_nodes, n_tris)) {
            active = false;
            finish(items[s]);
        }
    }
}

inline uint32_t blocks_for(uint64_t n, uint32_t b) { return (uint32_t)((n + b - 1) / b); }

struct TraceLaunch {
    DevScene s;
    const uint32_t* queue;
    const uint32_t* count;
    uint32_t* fetch;
    uint32_t max_n;
    const float4 *ro, *rd;
    float4* hit;
    const uint32_t* sh_id;
    const float4* sh_c;
    float4* rad;
    uint32_t* err;
    DevStats* stats;
    int kind;
    int sm_count;
    int bounce;
};

template <bool ANY, bool COUNT, int STACK>
void launch_one(const TraceLaunch& L, cudaStream_t st) {
    size_t smem = trace_smem<STACK>();
    if (SRT_TRACE_PERSISTENT && L.fetch) {
        uint32_t grid = (uint32_t)(L.sm_count > 0 ? L.sm_count : 148) * SRT_TRACE_PT_BLOCKS;
        grid = std::min(grid, std::max(1u, blocks_for(L.max_n, TRACE_BLOCK)));
        k_trace_pt<ANY, COUNT, STACK><<<grid, TRACE_BLOCK, smem, st>>>(L.s, L.queue, L.count, L.fetch, L.ro, L.rd,
                                                                      L.hit, L.sh_id, L.sh_c, L.rad, L.err, L.stats,
                                                                      L.kind, L.bounce);
    } else {
        k_trace<ANY, COUNT, STACK><<<blocks_for(L.max_n, TRACE_BLOCK), TRACE_BLOCK, smem, st>>>(
            L.s, L.queue, L.count, L.ro, L.rd, L.hit, L.sh_id, L.sh_c, L.rad, L.err, L.stats, L.kind, L.bounce);
    }
}

template <bool ANY>
void launch_kind(const TraceLaunch& L, int count_visits, cudaStream_t st) {
    bool small = L.s.depth <= (uint32_t)TRAV_STACK_SMALL;
    if (count_visits) {
        if (small) launch_one<ANY, true, TRAV_STACK_SMALL>(L, st);
        else launch_one<ANY, true, TRAV_STACK>(L, st);
    } else {
        if (small) launch_one<ANY, false, TRAV_STACK_SMALL>(L, st);
        else launch_one<ANY, false, TRAV_STACK>(L, st);
    }
}

}  // namespace

int launch_trace_closest(const FrameArgs& a, uint32_t bounce, cudaStream_t st) {
    // primary rays (bounce 0) are coherent (8 x 4 pixel tiles): one ray per
    // thread; later bounces are incoherent: persistent warps with refill
    TraceLaunch L{a.scene, a.pb.queue[bounce & 1], &a.counters->paths[bounce],
                  (bounce == 0 && !SRT_PRIMARY_PERSISTENT) ? nullptr : &a.counters->fetch[TRAV_CLOSEST][bounce],
                  a.width * a.height, a.pb.ray_o, a.pb.ray_d, a.pb.hit, nullptr, nullptr, nullptr, a.err, a.stats,
                  TRAV_CLOSEST, a.sm_count, (int)bounce};
    launch_kind<false>(L, a.count_visits, st);
    return 1;
}

int launch_trace_shadow(const FrameArgs& a, uint32_t bounce, cudaStream_t st) {
    // persistent warps with refill and pooled triangle tests (SRT_SHADOW_PERSISTENT_FROM)
    TraceLaunch L{a.scene, nullptr, &a.counters->shadow[bounce],
                  bounce >= (uint32_t)SRT_SHADOW_PERSISTENT_FROM
                      ? &a.counters->fetch[TRAV_SHADOW][bounce]
                      : nullptr,
                  a.width * a.height, a.pb.sh_o, a.pb.sh_d, nullptr, a.pb.sh_id, a.pb.sh_c, a.pb.rad, a.err, a.stats,
                  TRAV_SHADOW, a.sm_count, (int)bounce};
    launch_kind<true>(L, a.count_visits, st);
    return 1;
}

int launch_trace_queue(const DevScene& s, uint32_t bounce, const uint32_t* queue, const uint32_t* count,
                       uint32_t* fetch, uint32_t max_n, const float4* ro, const float4* rd, float4* hit, int kind,
                       int count_visits, uint32_t* err, DevStats* stats, int sm_count, cudaStream_t st) {
    if (max_n == 0) return 0;
    // photon rays in emitter order (direction-sorted with
    // SRT_PHOTON_DIR_SORT); persistent warps take them in that order
    // (SRT_PHOTON_PERSISTENT)
    TraceLaunch L{s, queue, count, SRT_PHOTON_PERSISTENT ? fetch : nullptr, max_n, ro, rd, hit, nullptr, nullptr,
                  nullptr, err, stats, kind, sm_count, (int)bounce};
    launch_kind<false>(L, count_visits, st);
    return 1;
}

int launch_trace_multi(const MultiTraceItem* items, int n_items, int any_hit, bool small_stack, uint32_t* fetch,
                       int blocks_per_sm, uint32_t chunk, int sm_count, cudaStream_t st) {
    if (n_items <= 0) return 0;
    uint32_t grid = (uint32_t)(sm_count > 0 ? sm_count : 148) * (uint32_t)std::max(1, blocks_per_sm);
    const int stack = small_stack ? TRAV_STACK_SMALL : TRAV_STACK;
    size_t smem = sizeof(uint2) * stack * TRACE_BLOCK;
    if (SRT_BATCH_TRACE_PT) {
        (void)chunk;
        if (any_hit) {
            if (small_stack) k_trace_multi_pt<true, TRAV_STACK_SMALL><<<grid, TRACE_BLOCK, smem, st>>>(items, n_items, fetch);
            else k_trace_multi_pt<true, TRAV_STACK><<<grid, TRACE_BLOCK, smem, st>>>(items, n_items, fetch);
        } else {
            if (small_stack) k_trace_multi_pt<false, TRAV_STACK_SMALL><<<grid, TRACE_BLOCK, smem, st>>>(items, n_items, fetch);
            else k_trace_multi_pt<false, TRAV_STACK><<<grid, TRACE_BLOCK, smem, st>>>(items, n_items, fetch);
        }
        return 1;
    }
    if (any_hit) {
        if (small_stack) k_trace_multi<true, TRAV_STACK_SMALL><<<grid, TRACE_BLOCK, smem, st>>>(items, n_items, fetch, chunk);
        else k_trace_multi<true, TRAV_STACK><<<grid, TRACE_BLOCK, smem, st>>>(items, n_items, fetch, chunk);
    } else {
        if (small_stack) k_trace_multi<false, TRAV_STACK_SMALL><<<grid, TRACE_BLOCK, smem, st>>>(items, n_items, fetch, chunk);
        else k_trace_multi<false, TRAV_STACK><<<grid, TRACE_BLOCK, smem, st>>>(items, n_items, fetch, chunk);
    }
    return 1;
}

int launch_trace_batch(const DevScene& s, const float4* rays, uint32_t n, float4* hits, int any_hit, uint32_t* err,
                       cudaStream_t st) {
    if (n == 0) return 0;
    size_t smem = sizeof(uint2) * TRAV_STACK * TRACE_BLOCK;
    if (any_hit)
        k_trace_batch<true><<<blocks_for(n, TRACE_BLOCK), TRACE_BLOCK, smem, st>>>(s, rays, n, hits, err);
    else
        k_trace_batch<false><<<blocks_for(n, TRACE_BLOCK), TRACE_BLOCK, smem, st>>>(s, rays, n, hits, err);
    return 1;
}

}  // namespace srt

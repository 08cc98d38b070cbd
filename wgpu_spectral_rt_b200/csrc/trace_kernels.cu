// trace_kernels.cu — closest-hit and any-hit wavefront kernels over the
// compressed BVH8 (the ray queries of shader.wgsl:561-566 and :654-659).
//
// Kept in their own translation unit: the traversal is compiled with
// multiply-add contraction (fast slab tests), while the shading kernels are
// compiled without it so that they round like the CPU oracle.
//
// The shared-memory stack is sized to the tree: STACK = 16 entries for trees
// of at most 16 levels (config 2 builds 10), 32 otherwise.
#include "render_kernels.h"

// 8 resident blocks of 128 threads per SM caps the kernels at 64 registers:
// the unbounded build takes ~110 and halves the warps in flight (measured:
// 8.7 ms vs 6.1 ms of closest-hit traversal per config-2 frame).
#ifndef SRT_TRACE_MIN_BLOCKS
#define SRT_TRACE_MIN_BLOCKS 8
#endif

namespace srt {

namespace {

template <bool ANY, bool COUNT, int STACK>
__global__ void __launch_bounds__(TRACE_BLOCK, SRT_TRACE_MIN_BLOCKS)
    k_trace(DevScene S, const uint32_t* __restrict__ queue, const uint32_t* __restrict__ count,
            const float4* __restrict__ ro, const float4* __restrict__ rd, float4* __restrict__ hit,
            const uint32_t* __restrict__ sh_id, const float4* __restrict__ sh_c, float4* __restrict__ rad,
            uint32_t* err, DevStats* stats, int kind) {
    extern __shared__ uint2 stack_smem[];
    uint32_t q = blockIdx.x * TRACE_BLOCK + threadIdx.x;
    uint32_t n = *count;
    if (q >= n) return;
    uint32_t id = queue ? queue[q] : q;
    float4 o = ro[ANY ? q : id], d = rd[ANY ? q : id];
    Ray ray{xyz(o), xyz(d), o.w, d.w};
    float t = 0.f, u = 0.f, v = 0.f;
    uint32_t prim;
    TravCounters tc{&stats->nodes_visited[kind], &stats->tris_tested[kind]};
    bool h = traverse<ANY, COUNT, STACK>(S, ray, stack_smem + threadIdx.x, TRACE_BLOCK, t, prim, u, v, err, tc);
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

inline uint32_t blocks_for(uint64_t n, uint32_t b) { return (uint32_t)((n + b - 1) / b); }

template <bool ANY, bool COUNT, int STACK>
void launch_k_trace(const FrameArgs& a, uint32_t bounce, cudaStream_t st) {
    uint32_t grid = blocks_for((uint64_t)a.width * a.height, TRACE_BLOCK);
    size_t smem = sizeof(uint2) * STACK * TRACE_BLOCK;
    if (ANY)
        k_trace<true, COUNT, STACK><<<grid, TRACE_BLOCK, smem, st>>>(a.scene, nullptr, &a.counters->shadow[bounce],
                                                                     a.pb.sh_o, a.pb.sh_d, nullptr, a.pb.sh_id,
                                                                     a.pb.sh_c, a.pb.rad, a.err, a.stats, TRAV_SHADOW);
    else
        k_trace<false, COUNT, STACK><<<grid, TRACE_BLOCK, smem, st>>>(a.scene, a.pb.queue[bounce & 1],
                                                                      &a.counters->paths[bounce], a.pb.ray_o,
                                                                      a.pb.ray_d, a.pb.hit, nullptr, nullptr, nullptr,
                                                                      a.err, a.stats, TRAV_CLOSEST);
}

template <bool COUNT, int STACK>
void launch_queue(const DevScene& s, const uint32_t* queue, const uint32_t* count, uint32_t max_n, const float4* ro,
                  const float4* rd, float4* hit, int kind, uint32_t* err, DevStats* stats, cudaStream_t st) {
    k_trace<false, COUNT, STACK><<<blocks_for(max_n, TRACE_BLOCK), TRACE_BLOCK, sizeof(uint2) * STACK * TRACE_BLOCK,
                                   st>>>(s, queue, count, ro, rd, hit, nullptr, nullptr, nullptr, err, stats, kind);
}

template <bool ANY>
void launch_trace_kind(const FrameArgs& a, uint32_t bounce, cudaStream_t st) {
    bool small = a.scene.depth <= (uint32_t)TRAV_STACK_SMALL;
    if (a.count_visits) {
        if (small) launch_k_trace<ANY, true, TRAV_STACK_SMALL>(a, bounce, st);
        else launch_k_trace<ANY, true, TRAV_STACK>(a, bounce, st);
    } else {
        if (small) launch_k_trace<ANY, false, TRAV_STACK_SMALL>(a, bounce, st);
        else launch_k_trace<ANY, false, TRAV_STACK>(a, bounce, st);
    }
}

}  // namespace

int launch_trace_closest(const FrameArgs& a, uint32_t bounce, cudaStream_t st) {
    launch_trace_kind<false>(a, bounce, st);
    return 1;
}

int launch_trace_shadow(const FrameArgs& a, uint32_t bounce, cudaStream_t st) {
    launch_trace_kind<true>(a, bounce, st);
    return 1;
}

int launch_trace_queue(const DevScene& s, const uint32_t* queue, const uint32_t* count, uint32_t max_n,
                       const float4* ro, const float4* rd, float4* hit, int kind, int count_visits, uint32_t* err,
                       DevStats* stats, cudaStream_t st) {
    if (max_n == 0) return 0;
    bool small = s.depth <= (uint32_t)TRAV_STACK_SMALL;
    if (count_visits) {
        if (small) launch_queue<true, TRAV_STACK_SMALL>(s, queue, count, max_n, ro, rd, hit, kind, err, stats, st);
        else launch_queue<true, TRAV_STACK>(s, queue, count, max_n, ro, rd, hit, kind, err, stats, st);
    } else {
        if (small) launch_queue<false, TRAV_STACK_SMALL>(s, queue, count, max_n, ro, rd, hit, kind, err, stats, st);
        else launch_queue<false, TRAV_STACK>(s, queue, count, max_n, ro, rd, hit, kind, err, stats, st);
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

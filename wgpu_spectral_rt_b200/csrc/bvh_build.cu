// bvh_build.cu — GPU build of the compressed 8-wide BVH over the scene's
// flattened world-space triangles.
//
// Replaces the driver's BLAS/TLAS build (src/scene/builder.rs:131-266).
// Instances are flattened (their triangles transformed to world space) so a
// single tree serves every ray; shading still uses the instance's object
// space data.  Steps, all on the device:
//   1. flatten: world-space triangle slots + per-triangle instance id
//   2. centroid bounds and 30-bit Morton codes
//   3. radix sort of (code, triangle) pairs
//   4. binary radix tree over the sorted codes (Karras, HPG 2012)
//   5. bottom-up bounding boxes (one thread per leaf, atomic visit flags)
//   6. collapse into 8-wide nodes, level by level: expand the child of
//      largest surface area until 8 children; subtrees of at most leaf_max
//      triangles (1..3, default 2) become leaves; children are placed in
//      slots by ray octant; child boxes are quantised to 8 bits against the
//      node's box.
#include <array>
#include <cmath>
#include <cstdio>
#include <string>
#include <vector>

#include "bvh_build.h"
#include "radix_sort.cuh"

namespace srt {

namespace {

constexpr uint32_t LEAF = 0x80000000u;
// A collapsed child with at most leaf_max triangles (BvhInputs) becomes a
// leaf (its triangles listed in the node); larger ones become 8-wide nodes.
// At most 3: a node's leaves share a 24-bit triangle mask and a 5-bit offset
// field.  The closest hit is the minimum of (t, id) and an any-hit answer does
// not depend on the order, so the choice changes speed, never results.
constexpr uint32_t LEAF_MAX_LIMIT = 3u;

__device__ __forceinline__ uint32_t float_flip(float f) {
    uint32_t u = __float_as_uint(f);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float float_unflip(uint32_t u) {
    return __uint_as_float((u & 0x80000000u) ? (u & 0x7FFFFFFFu) : ~u);
}

__global__ void k_flatten(const float4* __restrict__ vtx, const uint32_t* __restrict__ indices,
                          const uint4* __restrict__ mesh_infos, const InstDev* __restrict__ inst,
                          const InstFwd* __restrict__ fwd, uint32_t n_inst, uint32_t n_tris,
                          TriSlot* __restrict__ flat, uint32_t* __restrict__ tri_inst, float4* __restrict__ cen,
                          uint32_t* __restrict__ bounds /* 6 flipped: min xyz, max xyz */) {
    __shared__ uint32_t sb[6];
    if (threadIdx.x < 3) sb[threadIdx.x] = 0xFFFFFFFFu;
    else if (threadIdx.x < 6) sb[threadIdx.x] = 0u;
    __syncthreads();
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n_tris) {
        uint32_t lo = 0, hi = n_inst;  // last instance with tri_offset <= t
        while (hi - lo > 1) {
            uint32_t mid = (lo + hi) >> 1;
            if (inst[mid].tri_offset <= t) lo = mid;
            else hi = mid;
        }
        const InstDev& in = inst[lo];
        InstFwd f = fwd[lo];
        uint4 mi = mesh_infos[in.mesh_id];
        uint32_t io = mi.y + (t - in.tri_offset) * 3u;
        float3 w[3];
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            float4 p = vtx[2 * (indices[io + k] + mi.x)];
            w[k] = xform_point(f, p.x, p.y, p.z);
        }
        TriSlot s;
        s.v0 = make_float4(w[0].x, w[0].y, w[0].z, __uint_as_float(t));
        s.v1 = make_float4(w[1].x, w[1].y, w[1].z, 0.f);
        s.v2 = make_float4(w[2].x, w[2].y, w[2].z, 0.f);
        flat[t] = s;
        tri_inst[t] = lo;
        float3 c = (w[0] + w[1] + w[2]) * (1.0f / 3.0f);
        cen[t] = make_float4(c.x, c.y, c.z, 0.f);
        atomicMin(&sb[0], float_flip(c.x));
        atomicMin(&sb[1], float_flip(c.y));
        atomicMin(&sb[2], float_flip(c.z));
        atomicMax(&sb[3], float_flip(c.x));
        atomicMax(&sb[4], float_flip(c.y));
        atomicMax(&sb[5], float_flip(c.z));
    }
    __syncthreads();
    if (threadIdx.x < 3) atomicMin(&bounds[threadIdx.x], sb[threadIdx.x]);
    else if (threadIdx.x < 6) atomicMax(&bounds[threadIdx.x], sb[threadIdx.x]);
}

__device__ __forceinline__ uint32_t expand_bits(uint32_t v) {
    v = (v * 0x00010001u) & 0xFF0000FFu;
    v = (v * 0x00000101u) & 0x0F00F00Fu;
    v = (v * 0x00000011u) & 0xC30C30C3u;
    v = (v * 0x00000005u) & 0x49249249u;
    return v;
}

__global__ void k_morton(const float4* __restrict__ cen, const uint32_t* __restrict__ bounds, uint32_t n,
                         uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    float3 lo = f3(float_unflip(bounds[0]), float_unflip(bounds[1]), float_unflip(bounds[2]));
    float3 hi = f3(float_unflip(bounds[3]), float_unflip(bounds[4]), float_unflip(bounds[5]));
    float4 c = cen[t];
    float ex = fmaxf(hi.x - lo.x, 1e-30f), ey = fmaxf(hi.y - lo.y, 1e-30f), ez = fmaxf(hi.z - lo.z, 1e-30f);
    uint32_t x = (uint32_t)fminf(fmaxf((c.x - lo.x) / ex * 1024.0f, 0.0f), 1023.0f);
    uint32_t y = (uint32_t)fminf(fmaxf((c.y - lo.y) / ey * 1024.0f, 0.0f), 1023.0f);
    uint32_t z = (uint32_t)fminf(fmaxf((c.z - lo.z) / ez * 1024.0f, 0.0f), 1023.0f);
    keys[t] = (expand_bits(x) << 2) | (expand_bits(y) << 1) | expand_bits(z);
    vals[t] = t;
}

// delta(i, j): common prefix length of (key, index) pairs; -1 out of range.
__device__ __forceinline__ int delta(const uint32_t* keys, int n, int i, int j) {
    if (j < 0 || j >= n) return -1;
    uint32_t a = keys[i], b = keys[j];
    if (a == b) return 32 + __clz((uint32_t)i ^ (uint32_t)j);
    return __clz(a ^ b);
}

struct Bvh2 {
    uint4* inode;      // internal: left ref, right ref, first, last
    float4* ibox;      // internal: lo, hi (2 per node)
    float4* lbox;      // leaf: lo, hi
    uint32_t* iparent; // parent of internal node
    uint32_t* lparent; // parent of leaf
    uint32_t* flags;   // refit visit counters
};

__global__ void k_karras(const uint32_t* __restrict__ keys, int n, Bvh2 b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n - 1) return;
    int d = (delta(keys, n, i, i + 1) - delta(keys, n, i, i - 1)) >= 0 ? 1 : -1;
    int dmin = delta(keys, n, i, i - d);
    int lmax = 2;
    while (delta(keys, n, i, i + lmax * d) > dmin) lmax <<= 1;
    int l = 0;
    for (int t = lmax >> 1; t >= 1; t >>= 1)
        if (delta(keys, n, i, i + (l + t) * d) > dmin) l += t;
    int j = i + l * d;
    int dnode = delta(keys, n, i, j);
    int s = 0;
    int len = l;
    for (int t = (len + 1) >> 1;; t = (t + 1) >> 1) {
        if (delta(keys, n, i, i + (s + t) * d) > dnode) s += t;
        if (t == 1) break;
    }
    int gamma = i + s * d + min(d, 0);
    int first = min(i, j), last = max(i, j);
    uint32_t left = (first == gamma) ? (LEAF | (uint32_t)gamma) : (uint32_t)gamma;
    uint32_t right = (last == gamma + 1) ? (LEAF | (uint32_t)(gamma + 1)) : (uint32_t)(gamma + 1);
    b.inode[i] = make_uint4(left, right, (uint32_t)first, (uint32_t)last);
    if (left & LEAF) b.lparent[left & ~LEAF] = (uint32_t)i;
    else b.iparent[left] = (uint32_t)i;
    if (right & LEAF) b.lparent[right & ~LEAF] = (uint32_t)i;
    else b.iparent[right] = (uint32_t)i;
}

__global__ void k_refit(const TriSlot* __restrict__ flat, const uint32_t* __restrict__ sorted_tri, int n, Bvh2 b) {
    int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    TriSlot s = flat[sorted_tri[i]];
    float3 lo = f3(fminf(fminf(s.v0.x, s.v1.x), s.v2.x), fminf(fminf(s.v0.y, s.v1.y), s.v2.y),
                   fminf(fminf(s.v0.z, s.v1.z), s.v2.z));
    float3 hi = f3(fmaxf(fmaxf(s.v0.x, s.v1.x), s.v2.x), fmaxf(fmaxf(s.v0.y, s.v1.y), s.v2.y),
                   fmaxf(fmaxf(s.v0.z, s.v1.z), s.v2.z));
    b.lbox[2 * i] = make_float4(lo.x, lo.y, lo.z, 0.f);
    b.lbox[2 * i + 1] = make_float4(hi.x, hi.y, hi.z, 0.f);
    if (n == 1) return;
    uint32_t node = b.lparent[i];
    while (true) {
        __threadfence();
        if (atomicAdd(&b.flags[node], 1u) == 0u) return;  // the sibling finishes this node
        __threadfence();
        uint4 nd = b.inode[node];
        float4 a0, a1, c0, c1;
        if (nd.x & LEAF) {
            a0 = __ldcg(&b.lbox[2 * (nd.x & ~LEAF)]);
            a1 = __ldcg(&b.lbox[2 * (nd.x & ~LEAF) + 1]);
        } else {
            a0 = __ldcg(&b.ibox[2 * nd.x]);
            a1 = __ldcg(&b.ibox[2 * nd.x + 1]);
        }
        if (nd.y & LEAF) {
            c0 = __ldcg(&b.lbox[2 * (nd.y & ~LEAF)]);
            c1 = __ldcg(&b.lbox[2 * (nd.y & ~LEAF) + 1]);
        } else {
            c0 = __ldcg(&b.ibox[2 * nd.y]);
            c1 = __ldcg(&b.ibox[2 * nd.y + 1]);
        }
        b.ibox[2 * node] = make_float4(fminf(a0.x, c0.x), fminf(a0.y, c0.y), fminf(a0.z, c0.z), 0.f);
        b.ibox[2 * node + 1] = make_float4(fmaxf(a1.x, c1.x), fmaxf(a1.y, c1.y), fmaxf(a1.z, c1.z), 0.f);
        if (node == 0u) return;
        node = b.iparent[node];
    }
}

// ---------------------------------------------------------------- binned SAH
// Top-down, one level of the binary tree per round: every node still to be
// split (a task: a contiguous range of the primitive permutation) bins its
// primitives' centroids into SAH_BINS bins along its widest centroid axis,
// picks the bin boundary of least surface-area cost N_L A_L + N_R A_R (a
// median split by position when all centroids share one bin, and for every
// node below SAH_MEDIAN_LEVEL levels, which bounds the depth), and
// partitions its range.  The result is the same binary tree format as the
// LBVH (internal nodes over contiguous ranges, single-primitive leaves), so
// the bottom-up box pass and the 8-wide collapse are shared.
// Bins per axis: SAH_BINS for ranges binned with atomics in global memory
// (more than SAH_SMALL primitives), SAH_LOCAL_BINS for the small ranges that
// their split thread bins in a per-thread array (its stack frame, reserved for
// every resident thread, grows with the count: 3.0 KB at 16, 10.5 KB at 64).
// Config 2 (1.57M triangles, leaves of <= 2): 16 / 16 bins 7.80 node visits
// per camera ray, closest hits 3.00 ms per 1080p frame; 64 / 16 7.18 visits,
// 2.86 ms; 64 / 32 and 64 / 64 within noise of 64 / 16 (2.85, 2.83 ms), and
// 128 / 16 of 64 / 16 (2.87 vs 2.88 ms); 96 / 16 7.45 visits, 2.91 ms.  The
// same hits in every case: the tree changes speed, never results.
#ifndef SRT_SAH_BINS
#define SRT_SAH_BINS 64
#endif
#ifndef SRT_SAH_LOCAL_BINS
#define SRT_SAH_LOCAL_BINS 16
#endif
constexpr int SAH_BINS = SRT_SAH_BINS;
constexpr int SAH_LOCAL_BINS = SRT_SAH_LOCAL_BINS;
static_assert(SAH_LOCAL_BINS <= SAH_BINS, "bin counts");
constexpr int SAH_REC = 13;  // count, box lo/hi, centroid lo/hi (flipped floats)
constexpr int SAH_TASK_WORDS = 3 * SAH_BINS * SAH_REC;  // bins of the three axes
constexpr int SAH_LOCAL_WORDS = 3 * SAH_LOCAL_BINS * SAH_REC;
constexpr uint32_t SAH_MEDIAN = 0xFFFFFFFFu;
constexpr uint32_t SAH_LOCAL = 0xFFFFFFFEu;  // binned by its split thread (small ranges)
constexpr uint32_t SAH_SMALL = 64;           // ranges up to this size bin without atomics
constexpr uint32_t SAH_MEDIAN_LEVEL = 48;

struct SahTask {
    uint32_t node, first, count, axis;
    float cmin[3], cscale[3];  // bin along axis a = (c_a - cmin[a]) * cscale[a]
    uint32_t nbins;            // bins per axis: SAH_BINS, or SAH_LOCAL_BINS for small ranges
    uint32_t bin_slot;         // bins of this task (SAH tasks only)
    uint32_t split, left_count;
    uint32_t lcur, rcur;
    uint32_t child_task[2];  // next-level task of each child, 0xFFFFFFFF for a leaf
};

__device__ __forceinline__ uint32_t sah_bin(const SahTask& t, float4 c, uint32_t ax) {
    float v = ax == 0 ? c.x : (ax == 1 ? c.y : c.z);
    float f = (v - t.cmin[ax]) * t.cscale[ax];
    int b = (int)f;
    return (uint32_t)min(max(b, 0), (int)t.nbins - 1);
}

__device__ __forceinline__ uint32_t sah_init_word(uint32_t i) {
    uint32_t k = i % SAH_REC;
    // lo fields start at +inf (min of flipped), hi fields at 0
    return (k == 0u) ? 0u : ((k >= 1 && k <= 3) || (k >= 7 && k <= 9)) ? 0xFFFFFFFFu : 0u;
}

__global__ void k_sah_init_bins(uint32_t* __restrict__ bins, uint32_t n_words) {
    uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_words) return;
    bins[i] = sah_init_word(i);
}

__device__ __forceinline__ void sah_accum(uint32_t* rec, float3 lo, float3 hi, float4 c) {
    atomicAdd(&rec[0], 1u);
    atomicMin(&rec[1], float_flip(lo.x));
    atomicMin(&rec[2], float_flip(lo.y));
    atomicMin(&rec[3], float_flip(lo.z));
    atomicMax(&rec[4], float_flip(hi.x));
    atomicMax(&rec[5], float_flip(hi.y));
    atomicMax(&rec[6], float_flip(hi.z));
    atomicMin(&rec[7], float_flip(c.x));
    atomicMin(&rec[8], float_flip(c.y));
    atomicMin(&rec[9], float_flip(c.z));
    atomicMax(&rec[10], float_flip(c.x));
    atomicMax(&rec[11], float_flip(c.y));
    atomicMax(&rec[12], float_flip(c.z));
}

// Bins of every active position (of tasks larger than SAH_SMALL) along all
// three axes; the tasks of the block's first and last positions (most of the
// block) aggregate in shared memory.
__global__ void k_sah_bin(const uint32_t* __restrict__ perm, const int* __restrict__ pos_task, uint32_t n,
                          const SahTask* __restrict__ tasks, const float4* __restrict__ cen,
                          const TriSlot* __restrict__ flat, uint32_t* __restrict__ bins) {
    __shared__ uint32_t sb[2][SAH_TASK_WORDS];
    __shared__ int ts[2];
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (threadIdx.x == 0) {
        ts[0] = pos_task[min(blockIdx.x * blockDim.x, n - 1)];
        ts[1] = pos_task[min(blockIdx.x * blockDim.x + blockDim.x - 1, n - 1)];
        if (ts[1] == ts[0]) ts[1] = -1;
        for (int k = 0; k < 2; ++k)
            if (ts[k] >= 0 && tasks[ts[k]].split != 0u) ts[k] = -1;
    }
    for (int i = threadIdx.x; i < 2 * SAH_TASK_WORDS; i += blockDim.x)
        sb[i / SAH_TASK_WORDS][i % SAH_TASK_WORDS] = sah_init_word((uint32_t)(i % SAH_TASK_WORDS));
    __syncthreads();
    if (p < n) {
        const int t = pos_task[p];
        if (t >= 0 && tasks[t].split == 0u) {
            const SahTask& T = tasks[t];
            const uint32_t prim = perm[p];
            const TriSlot s = flat[prim];
            const float3 lo = f3(fminf(fminf(s.v0.x, s.v1.x), s.v2.x), fminf(fminf(s.v0.y, s.v1.y), s.v2.y),
                                 fminf(fminf(s.v0.z, s.v1.z), s.v2.z));
            const float3 hi = f3(fmaxf(fmaxf(s.v0.x, s.v1.x), s.v2.x), fmaxf(fmaxf(s.v0.y, s.v1.y), s.v2.y),
                                 fmaxf(fmaxf(s.v0.z, s.v1.z), s.v2.z));
            const float4 c = cen[prim];
            uint32_t* dst = t == ts[0] ? sb[0] : t == ts[1] ? sb[1] : bins + (size_t)T.bin_slot * SAH_TASK_WORDS;
            for (uint32_t ax = 0; ax < 3; ++ax) {
                if (!(T.cscale[ax] > 0.f)) continue;
                sah_accum(dst + (ax * SAH_BINS + sah_bin(T, c, ax)) * SAH_REC, lo, hi, c);
            }
        }
    }
    __syncthreads();
    for (int k = 0; k < 2; ++k) {
        if (ts[k] < 0) continue;
        uint32_t* G = bins + (size_t)tasks[ts[k]].bin_slot * SAH_TASK_WORDS;
        for (int i = threadIdx.x; i < 3 * SAH_BINS; i += blockDim.x) {
            const uint32_t* r = sb[k] + i * SAH_REC;
            if (r[0] == 0u) continue;
            uint32_t* g = G + i * SAH_REC;
            atomicAdd(&g[0], r[0]);
            for (int j = 1; j <= 3; ++j) atomicMin(&g[j], r[j]);
            for (int j = 4; j <= 6; ++j) atomicMax(&g[j], r[j]);
            for (int j = 7; j <= 9; ++j) atomicMin(&g[j], r[j]);
            for (int j = 10; j <= 12; ++j) atomicMax(&g[j], r[j]);
        }
    }
}

__device__ __forceinline__ float half_area(float3 lo, float3 hi) {
    float3 e = f3(fmaxf(hi.x - lo.x, 0.f), fmaxf(hi.y - lo.y, 0.f), fmaxf(hi.z - lo.z, 0.f));
    return e.x * e.y + e.y * e.z + e.z * e.x;
}

// Sets the next-level task of one child: bin mappings of the three axes from
// its centroid bounds, and a bin slot when it will be binned.
__device__ void sah_child_task(SahTask& c, uint32_t node, uint32_t first, uint32_t count, float3 clo, float3 chi,
                               bool median, uint32_t* bin_alloc, uint32_t bin_cap) {
    c.node = node;
    c.first = first;
    c.count = count;
    const float lo[3] = {clo.x, clo.y, clo.z}, ext[3] = {chi.x - clo.x, chi.y - clo.y, chi.z - clo.z};
    bool any = false;
    for (int a = 0; a < 3; ++a) {
        c.cmin[a] = lo[a];
        c.cscale[a] = ext[a] > 0.f ? (float)(count <= SAH_SMALL ? SAH_LOCAL_BINS : SAH_BINS) / ext[a] : 0.f;
        any = any || ext[a] > 0.f;
    }
    c.axis = 0;
    c.nbins = count <= SAH_SMALL ? (uint32_t)SAH_LOCAL_BINS : (uint32_t)SAH_BINS;
    // all centroids on one point, below the SAH levels, or a range that the
    // collapse turns into one leaf anyway (<= 3): split by position
    c.split = (median || !any || count <= 3u) ? SAH_MEDIAN : (count <= SAH_SMALL ? SAH_LOCAL : 0u);
    c.bin_slot = 0xFFFFFFFFu;
    if (c.split == 0u) {
        uint32_t slot = atomicAdd(bin_alloc, 1u);
        if (slot < bin_cap) c.bin_slot = slot;
        else c.split = SAH_MEDIAN;  // out of bin slots (cannot happen: n / (SAH_SMALL + 1) tasks)
    }
    c.left_count = 0;
    c.lcur = c.rcur = 0;
    c.child_task[0] = c.child_task[1] = 0xFFFFFFFFu;
}

// One thread per task: choose the split (axis and bin boundary of least
// cost), create the children.
__global__ void k_sah_split(SahTask* __restrict__ tasks, uint32_t n_tasks, const uint32_t* __restrict__ bins,
                            const uint32_t* __restrict__ perm, const float4* __restrict__ cen,
                            const TriSlot* __restrict__ flat,
                            SahTask* __restrict__ next, uint32_t* __restrict__ n_next, uint32_t next_cap,
                            uint32_t* __restrict__ bin_alloc, uint32_t bin_cap, uint32_t* __restrict__ node_alloc,
                            uint32_t node_cap, Bvh2 b, uint32_t level, uint32_t* __restrict__ err) {
    const uint32_t ti = blockIdx.x * blockDim.x + threadIdx.x;
    if (ti >= n_tasks) return;
    SahTask& T = tasks[ti];
    uint32_t left = T.count / 2;  // median by position
    float3 clo[2] = {f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f)}, chi[2] = {f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f)};
    bool median = T.split == SAH_MEDIAN;
    uint32_t local[SAH_LOCAL_WORDS];  // the bins of a small range, filled here without atomics
    const uint32_t* Bt = local;
    if (T.split == 0u) Bt = bins + (size_t)T.bin_slot * SAH_TASK_WORDS;
    if (T.split == SAH_LOCAL) {
        for (int i = 0; i < SAH_LOCAL_WORDS; ++i) local[i] = sah_init_word((uint32_t)i);
        for (uint32_t q = T.first; q < T.first + T.count; ++q) {
            const uint32_t prim = perm[q];
            const TriSlot s = flat[prim];
            const float4 c = cen[prim];
            const uint32_t f[12] = {float_flip(fminf(fminf(s.v0.x, s.v1.x), s.v2.x)),
                                    float_flip(fminf(fminf(s.v0.y, s.v1.y), s.v2.y)),
                                    float_flip(fminf(fminf(s.v0.z, s.v1.z), s.v2.z)),
                                    float_flip(fmaxf(fmaxf(s.v0.x, s.v1.x), s.v2.x)),
                                    float_flip(fmaxf(fmaxf(s.v0.y, s.v1.y), s.v2.y)),
                                    float_flip(fmaxf(fmaxf(s.v0.z, s.v1.z), s.v2.z)),
                                    float_flip(c.x), float_flip(c.y), float_flip(c.z),
                                    float_flip(c.x), float_flip(c.y), float_flip(c.z)};
            for (uint32_t ax = 0; ax < 3; ++ax) {
                if (!(T.cscale[ax] > 0.f)) continue;
                uint32_t* r = local + (ax * SAH_LOCAL_BINS + sah_bin(T, c, ax)) * SAH_REC;
                r[0] += 1u;
                for (int j = 0; j < 3; ++j) {
                    r[1 + j] = min(r[1 + j], f[j]);
                    r[4 + j] = max(r[4 + j], f[3 + j]);
                    r[7 + j] = min(r[7 + j], f[6 + j]);
                    r[10 + j] = max(r[10 + j], f[9 + j]);
                }
            }
        }
        T.split = 0u;
    }
    if (!median) {
        float best = 3.4e38f;
        int bk = -1, bax = -1;
        const int NB = (int)T.nbins;  // the bin arrays' stride per axis
        for (int ax = 0; ax < 3; ++ax) {
            if (!(T.cscale[ax] > 0.f)) continue;
            const uint32_t* B = Bt + ax * NB * SAH_REC;
            float ra[SAH_BINS];  // area of bins [k, K)
            uint32_t rc[SAH_BINS];
            float3 lo = f3(3.4e38f, 3.4e38f, 3.4e38f), hi = f3(-3.4e38f, -3.4e38f, -3.4e38f);
            uint32_t cnt = 0;
            for (int k = NB - 1; k >= 0; --k) {
                const uint32_t* r = B + k * SAH_REC;
                if (r[0]) {
                    lo = f3(fminf(lo.x, float_unflip(r[1])), fminf(lo.y, float_unflip(r[2])),
                            fminf(lo.z, float_unflip(r[3])));
                    hi = f3(fmaxf(hi.x, float_unflip(r[4])), fmaxf(hi.y, float_unflip(r[5])),
                            fmaxf(hi.z, float_unflip(r[6])));
                    cnt += r[0];
                }
                ra[k] = cnt ? half_area(lo, hi) : 0.f;
                rc[k] = cnt;
            }
            lo = f3(3.4e38f, 3.4e38f, 3.4e38f);
            hi = f3(-3.4e38f, -3.4e38f, -3.4e38f);
            cnt = 0;
            for (int k = 1; k < NB; ++k) {
                const uint32_t* r = B + (k - 1) * SAH_REC;
                if (r[0]) {
                    lo = f3(fminf(lo.x, float_unflip(r[1])), fminf(lo.y, float_unflip(r[2])),
                            fminf(lo.z, float_unflip(r[3])));
                    hi = f3(fmaxf(hi.x, float_unflip(r[4])), fmaxf(hi.y, float_unflip(r[5])),
                            fmaxf(hi.z, float_unflip(r[6])));
                    cnt += r[0];
                }
                if (cnt == 0 || rc[k] == 0) continue;
                float cost = (float)cnt * half_area(lo, hi) + (float)rc[k] * ra[k];
                if (cost < best) {
                    best = cost;
                    bk = k;
                    bax = ax;
                }
            }
        }
        if (bk < 0) {
            median = true;
        } else {
            T.axis = (uint32_t)bax;
            T.split = (uint32_t)bk;
            left = 0;
            const uint32_t* B = Bt + bax * NB * SAH_REC;
            float3 l0 = f3(3.4e38f, 3.4e38f, 3.4e38f), h0 = f3(-3.4e38f, -3.4e38f, -3.4e38f), l1 = l0, h1 = h0;
            for (int k = 0; k < NB; ++k) {
                const uint32_t* r = B + k * SAH_REC;
                if (!r[0]) continue;
                float3 a = f3(float_unflip(r[7]), float_unflip(r[8]), float_unflip(r[9]));
                float3 z = f3(float_unflip(r[10]), float_unflip(r[11]), float_unflip(r[12]));
                if (k < bk) {
                    left += r[0];
                    l0 = f3(fminf(l0.x, a.x), fminf(l0.y, a.y), fminf(l0.z, a.z));
                    h0 = f3(fmaxf(h0.x, z.x), fmaxf(h0.y, z.y), fmaxf(h0.z, z.z));
                } else {
                    l1 = f3(fminf(l1.x, a.x), fminf(l1.y, a.y), fminf(l1.z, a.z));
                    h1 = f3(fmaxf(h1.x, z.x), fmaxf(h1.y, z.y), fmaxf(h1.z, z.z));
                }
            }
            clo[0] = l0;
            chi[0] = h0;
            clo[1] = l1;
            chi[1] = h1;
        }
    }
    if (median) {
        T.split = SAH_MEDIAN;
        left = T.count / 2;
        // centroid bounds are not tracked for position splits: the children
        // keep splitting by position
    }
    T.left_count = left;
    const uint32_t firsts[2] = {T.first, T.first + left}, counts[2] = {left, T.count - left};
    uint32_t refs[2];
    for (int c = 0; c < 2; ++c) {
        if (counts[c] == 1u) {
            refs[c] = LEAF | firsts[c];
            b.lparent[firsts[c]] = T.node;
            T.child_task[c] = 0xFFFFFFFFu;
        } else {
            uint32_t nd = atomicAdd(node_alloc, 1u);
            uint32_t tn = atomicAdd(n_next, 1u);
            if (nd >= node_cap || tn >= next_cap || counts[c] == 0u) {
                atomicOr(err, ERR_QUEUE_OVERFLOW);
                refs[c] = 0u;
                T.child_task[c] = 0xFFFFFFFFu;
                continue;
            }
            refs[c] = nd;
            b.iparent[nd] = T.node;
            T.child_task[c] = tn;
            sah_child_task(next[tn], nd, firsts[c], counts[c], clo[c], chi[c], median || level + 1 >= SAH_MEDIAN_LEVEL,
                           bin_alloc, bin_cap);
        }
    }
    b.inode[T.node] = make_uint4(refs[0], refs[1], T.first, T.first + T.count - 1u);
}

__global__ void k_sah_root(const uint32_t* __restrict__ bounds, uint32_t n, SahTask* __restrict__ t,
                           int* __restrict__ pos_task, uint32_t* __restrict__ perm, uint32_t* __restrict__ bin_alloc,
                           uint32_t bin_cap) {
    uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p == 0) {
        float3 lo = f3(float_unflip(bounds[0]), float_unflip(bounds[1]), float_unflip(bounds[2]));
        float3 hi = f3(float_unflip(bounds[3]), float_unflip(bounds[4]), float_unflip(bounds[5]));
        sah_child_task(t[0], 0u, 0u, n, lo, hi, false, bin_alloc, bin_cap);
    }
    if (p < n) {
        pos_task[p] = 0;
        perm[p] = p;
    }
}

// Moves every active primitive into its child's range.
__global__ void k_sah_partition(const uint32_t* __restrict__ perm, const int* __restrict__ pos_task, uint32_t n,
                                SahTask* __restrict__ tasks, const float4* __restrict__ cen,
                                uint32_t* __restrict__ perm2, int* __restrict__ pos_task2) {
    const uint32_t p = blockIdx.x * blockDim.x + threadIdx.x;
    if (p >= n) return;
    const int t = pos_task[p];
    const uint32_t prim = perm[p];
    if (t < 0) {
        perm2[p] = prim;
        pos_task2[p] = -1;
        return;
    }
    SahTask& T = tasks[t];
    uint32_t side;
    if (T.split == SAH_MEDIAN) side = (p - T.first) >= T.left_count ? 1u : 0u;
    else side = sah_bin(T, cen[prim], T.axis) >= T.split ? 1u : 0u;
    uint32_t np = side ? T.first + T.left_count + atomicAdd(&T.rcur, 1u) : T.first + atomicAdd(&T.lcur, 1u);
    perm2[np] = prim;
    pos_task2[np] = T.child_task[side] == 0xFFFFFFFFu ? -1 : (int)T.child_task[side];
}

__device__ __forceinline__ void ref_box(const Bvh2& b, uint32_t r, float3& lo, float3& hi) {
    float4 a, c;
    if (r & LEAF) {
        a = b.lbox[2 * (r & ~LEAF)];
        c = b.lbox[2 * (r & ~LEAF) + 1];
    } else {
        a = b.ibox[2 * r];
        c = b.ibox[2 * r + 1];
    }
    lo = xyz(a);
    hi = xyz(c);
}
__device__ __forceinline__ void ref_range(const Bvh2& b, uint32_t r, uint32_t& first, uint32_t& count) {
    if (r & LEAF) {
        first = r & ~LEAF;
        count = 1;
    } else {
        uint4 nd = b.inode[r];
        first = nd.z;
        count = nd.w - nd.z + 1;
    }
}

// Quantisation frame and 8-bit child boxes of one node, children indexed by
// slot (slots outside `used` empty): writes nd.a (origin, exponent bytes,
// imask), nd.c, nd.d, nd.e.  250 quanta span the node; the origin sits two
// quanta below it, and every child plane is padded outward by one quantum,
// which covers the half-quantum error of the traversal's biased-byte
// evaluation (see traverse<> in device_common.cuh).
__device__ void quantize_node(float3 nlo, float3 nhi, const float3* slo, const float3* shi, uint32_t used,
                              uint32_t imask, Node8& nd, uint32_t* err) {
    uint32_t ebyte[3];
    float scale[3];
    float nlov[3] = {nlo.x, nlo.y, nlo.z}, nhiv[3] = {nhi.x, nhi.y, nhi.z};
    for (int a = 0; a < 3; ++a) {
        double ext = (double)nhiv[a] - (double)nlov[a];
        int ex = -126;
        if (ext > 0.0) {
            ex = (int)ceil(log2(ext / 250.0));
            if (ldexp(250.0, ex) < ext) ++ex;
        }
        // a quantum of at least 4 float ulps of the node's coordinates, so the
        // shifted origin below stays exact to a quarter quantum
        double mag = fmax(fabs((double)nlov[a]), fabs((double)nhiv[a]));
        ex = max(ex, (int)ceil(log2(fmax(mag, 1e-30) * 4.0 / 8388608.0)));
        ex = max(ex, -126);
        ex = min(ex, 127);
        ebyte[a] = (uint32_t)(ex + 127);
        scale[a] = __uint_as_float(ebyte[a] << 23);
        double lo_exact = (double)nlov[a];
        nlov[a] = (float)(lo_exact - 2.0 * (double)scale[a]);
        while ((double)nlov[a] > lo_exact - 2.0 * (double)scale[a]) nlov[a] = nextafterf(nlov[a], -3.4e38f);
    }
    uint32_t qlo[3][2] = {{0u, 0u}, {0u, 0u}, {0u, 0u}}, qhi[3][2] = {{0u, 0u}, {0u, 0u}, {0u, 0u}};
    for (int s = 0; s < 8; ++s) {
        if (!((used >> s) & 1u)) continue;
        float lo3[3] = {slo[s].x, slo[s].y, slo[s].z}, hi3[3] = {shi[s].x, shi[s].y, shi[s].z};
        for (int a = 0; a < 3; ++a) {
            double sc = (double)scale[a];
            // one quantum of padding on each side
            int ql = (int)floor(((double)lo3[a] - (double)nlov[a]) / sc) - 1;
            int qh = (int)ceil(((double)hi3[a] - (double)nlov[a]) / sc) + 1;
            ql = min(max(ql, 0), 255);
            qh = min(max(qh, 0), 255);
            while (ql > 0 && (double)nlov[a] + ql * sc > (double)lo3[a] - sc) --ql;
            while (qh < 255 && (double)nlov[a] + qh * sc < (double)hi3[a] + sc) ++qh;
            if ((double)nlov[a] + ql * sc > (double)lo3[a] - sc || (double)nlov[a] + qh * sc < (double)hi3[a] + sc)
                atomicOr(err, ERR_BAD_INDEX);  // the frame cannot hold the padded child: reject the tree
            qlo[a][s >> 2] |= (uint32_t)ql << (8 * (s & 3));
            qhi[a][s >> 2] |= (uint32_t)qh << (8 * (s & 3));
        }
    }
    nd.a = make_uint4(__float_as_uint(nlov[0]), __float_as_uint(nlov[1]), __float_as_uint(nlov[2]),
                      ebyte[0] | (ebyte[1] << 8) | (ebyte[2] << 16) | (imask << 24));
    nd.c = make_uint4(qlo[0][0], qlo[0][1], qlo[1][0], qlo[1][1]);
    nd.d = make_uint4(qlo[2][0], qlo[2][1], qhi[0][0], qhi[0][1]);
    nd.e = make_uint4(qhi[1][0], qhi[1][1], qhi[2][0], qhi[2][1]);
}

// Refit of one level's nodes: child boxes from the deeper level's results
// (aux) or from the leaf triangles, then the node's frame is re-quantised.
__global__ void k_refit8(Node8* __restrict__ nodes, const TriSlot* __restrict__ tris, uint32_t begin, uint32_t end,
                         float4* __restrict__ aux, uint32_t* __restrict__ err) {
    uint32_t i = begin + blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= end) return;
    Node8 nd = nodes[i];
    const uint32_t imask = nd.a.w >> 24, child_base = nd.b.x, tri_base = nd.b.y;
    const uint32_t meta[2] = {nd.b.z, nd.b.w};
    float3 slo[8], shi[8];
    float3 nlo = f3(3.4e38f, 3.4e38f, 3.4e38f), nhi = f3(-3.4e38f, -3.4e38f, -3.4e38f);
    uint32_t used = 0u;
    for (int s = 0; s < 8; ++s) {
        const uint32_t m = (meta[s >> 2] >> (8 * (s & 3))) & 0xFFu;
        if (m == 0u) continue;
        used |= 1u << s;
        float3 lo, hi;
        if ((imask >> s) & 1u) {
            const uint32_t child = child_base + __popc(imask & ((1u << s) - 1u));
            float4 a = aux[2 * child], b = aux[2 * child + 1];
            lo = f3(a.x, a.y, a.z);
            hi = f3(b.x, b.y, b.z);
        } else {
            lo = f3(3.4e38f, 3.4e38f, 3.4e38f);
            hi = f3(-3.4e38f, -3.4e38f, -3.4e38f);
            const uint32_t cnt = m >> 5, off = m & 31u;
            for (uint32_t k = 0; k < cnt; ++k) {
                const TriSlot& t = tris[tri_base + off + k];
                float3 v[3] = {f3(t.v0.x, t.v0.y, t.v0.z), f3(t.v1.x, t.v1.y, t.v1.z), f3(t.v2.x, t.v2.y, t.v2.z)};
                for (int j = 0; j < 3; ++j) {
                    lo = f3(fminf(lo.x, v[j].x), fminf(lo.y, v[j].y), fminf(lo.z, v[j].z));
                    hi = f3(fmaxf(hi.x, v[j].x), fmaxf(hi.y, v[j].y), fmaxf(hi.z, v[j].z));
                }
            }
        }
        slo[s] = lo;
        shi[s] = hi;
        nlo = f3(fminf(nlo.x, lo.x), fminf(nlo.y, lo.y), fminf(nlo.z, lo.z));
        nhi = f3(fmaxf(nhi.x, hi.x), fmaxf(nhi.y, hi.y), fmaxf(nhi.z, hi.z));
    }
    aux[2 * i] = make_float4(nlo.x, nlo.y, nlo.z, 0.f);
    aux[2 * i + 1] = make_float4(nhi.x, nhi.y, nhi.z, 0.f);
    quantize_node(nlo, nhi, slo, shi, used, imask, nd, err);
    nodes[i] = nd;
}

// Leaf slots of moved instances, re-transformed from object space.
__global__ void k_update_slots(TriSlot* __restrict__ tris, uint32_t n_tris, const uint32_t* __restrict__ tri_inst,
                               const uint8_t* __restrict__ moved, const float4* __restrict__ vtx,
                               const uint32_t* __restrict__ indices, const uint4* __restrict__ mesh_infos,
                               const InstDev* __restrict__ inst, const InstFwd* __restrict__ fwd) {
    uint32_t k = blockIdx.x * blockDim.x + threadIdx.x;
    if (k >= n_tris) return;
    TriSlot s = tris[k];
    const uint32_t t = __float_as_uint(s.v0.w);
    const uint32_t ii = tri_inst[t];
    if (!moved[ii]) return;
    const InstDev& in = inst[ii];
    const InstFwd f = fwd[ii];
    const uint4 mi = mesh_infos[in.mesh_id];
    const uint32_t io = mi.y + (t - in.tri_offset) * 3u;
    float3 w[3];
    for (int j = 0; j < 3; ++j) {
        float4 p = vtx[2 * (indices[io + j] + mi.x)];
        w[j] = xform_point(f, p.x, p.y, p.z);
    }
    s.v0 = make_float4(w[0].x, w[0].y, w[0].z, s.v0.w);
    s.v1 = make_float4(w[1].x, w[1].y, w[1].z, 0.f);
    s.v2 = make_float4(w[2].x, w[2].y, w[2].z, 0.f);
    tris[k] = s;
}

// One block per light instance: its triangles in world space
// (builder.rs:101-129; w = 1, params copied).
__global__ void k_expand_lights(const LightInst* __restrict__ li, const uint8_t* __restrict__ moved,
                                const float4* __restrict__ vtx, const uint32_t* __restrict__ indices,
                                const uint4* __restrict__ mesh_infos, const InstDev* __restrict__ inst,
                                const InstFwd* __restrict__ fwd, float4* __restrict__ lights) {
    const LightInst L = li[blockIdx.x];
    if (moved && !moved[L.inst]) return;
    const InstDev& in = inst[L.inst];
    const InstFwd f = fwd[L.inst];
    const uint4 mi = mesh_infos[in.mesh_id];
    for (uint32_t k = threadIdx.x; k < L.count; k += blockDim.x) {
        float4* o = lights + 4ull * (L.first + k);
        for (int j = 0; j < 3; ++j) {
            float4 p = vtx[2 * (indices[mi.y + 3u * k + j] + mi.x)];
            float3 w = xform_point(f, p.x, p.y, p.z);
            o[j] = make_float4(w.x, w.y, w.z, 1.0f);
        }
        o[3] = L.params;
    }
}

// One thread per 8-wide node of this level: queue entries (bvh2 ref, node).
__global__ void k_collapse(Bvh2 b, const uint2* __restrict__ qin, uint32_t n_in, uint2* __restrict__ qout,
                           uint32_t* __restrict__ n_out, Node8* __restrict__ nodes, uint32_t* __restrict__ node_alloc,
                           uint32_t node_cap, TriSlot* __restrict__ tris_out, uint32_t* __restrict__ tri_alloc,
                           uint32_t tri_cap, const TriSlot* __restrict__ flat, const uint32_t* __restrict__ sorted_tri,
                           uint32_t* __restrict__ err, int width, uint32_t leaf_max) {
    uint32_t e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= n_in) return;
    uint2 q = qin[e];
    uint32_t refs[8];
    int nc;
    if (q.x & LEAF) {
        refs[0] = q.x;
        nc = 1;
    } else {
        uint4 nd = b.inode[q.x];
        refs[0] = nd.x;
        refs[1] = nd.y;
        nc = 2;
    }
    while (nc < width) {
        int best = -1;
        float best_area = -1.0f;
        for (int c = 0; c < nc; ++c) {
            if (refs[c] & LEAF) continue;
            float3 lo, hi;
            ref_box(b, refs[c], lo, hi);
            float3 ext = hi - lo;
            float area = ext.x * ext.y + ext.y * ext.z + ext.z * ext.x;
            if (area > best_area) {
                best_area = area;
                best = c;
            }
        }
        if (best < 0) break;
        uint4 nd = b.inode[refs[best]];
        refs[best] = nd.x;
        refs[nc++] = nd.y;
    }
    // children boxes, counts and node box
    float3 clo[8], chi[8];
    uint32_t cfirst[8], ccount[8];
    float3 nlo = f3(3.4e38f, 3.4e38f, 3.4e38f), nhi = f3(-3.4e38f, -3.4e38f, -3.4e38f);
    uint32_t n_int = 0, n_tri = 0;
    for (int c = 0; c < nc; ++c) {
        ref_box(b, refs[c], clo[c], chi[c]);
        ref_range(b, refs[c], cfirst[c], ccount[c]);
        nlo = f3(fminf(nlo.x, clo[c].x), fminf(nlo.y, clo[c].y), fminf(nlo.z, clo[c].z));
        nhi = f3(fmaxf(nhi.x, chi[c].x), fmaxf(nhi.y, chi[c].y), fmaxf(nhi.z, chi[c].z));
        if (ccount[c] <= leaf_max) n_tri += ccount[c];
        else ++n_int;
    }
    uint32_t child_base = n_int ? atomicAdd(node_alloc, n_int) : 0u;
    uint32_t tri_base = n_tri ? atomicAdd(tri_alloc, n_tri) : 0u;
    if (child_base + n_int > node_cap || tri_base + n_tri > tri_cap) {
        atomicOr(err, ERR_QUEUE_OVERFLOW);
        return;
    }
    // slot assignment: slot s is visited first by rays whose octant is s
    // (bit set = negative direction), which want the child lying farthest
    // along +x/+y/+z for set bits; greedy on the best (child, slot) score.
    float3 pc = (nlo + nhi) * 0.5f;
    int slot_of[8];
    int child_in[8];
    for (int s = 0; s < 8; ++s) child_in[s] = -1;
    for (int c = 0; c < nc; ++c) slot_of[c] = -1;
    for (int it = 0; it < nc; ++it) {
        float bs = -3.4e38f;
        int bc = -1, bsl = -1;
        for (int c = 0; c < nc; ++c) {
            if (slot_of[c] >= 0) continue;
            float3 d = (clo[c] + chi[c]) * 0.5f - pc;
            for (int s = 0; s < 8; ++s) {
                if (child_in[s] >= 0) continue;
                float sc = ((s & 1) ? d.x : -d.x) + ((s & 2) ? d.y : -d.y) + ((s & 4) ? d.z : -d.z);
                if (sc > bs) {
                    bs = sc;
                    bc = c;
                    bsl = s;
                }
            }
        }
        slot_of[bc] = bsl;
        child_in[bsl] = bc;
    }
    uint32_t meta[2] = {0u, 0u};
    uint32_t imask = 0u, int_rank = 0u, tri_off = 0u, used = 0u;
    float3 slo[8], shi[8];
    for (int s = 0; s < 8; ++s) {
        int c = child_in[s];
        if (c < 0) continue;
        used |= 1u << s;
        slo[s] = clo[c];
        shi[s] = chi[c];
        uint32_t m;
        if (ccount[c] <= leaf_max) {
            m = (ccount[c] << 5) | tri_off;
            for (uint32_t k = 0; k < ccount[c]; ++k) tris_out[tri_base + tri_off + k] = flat[sorted_tri[cfirst[c] + k]];
            tri_off += ccount[c];
        } else {
            m = 7u << 5;
            imask |= 1u << s;
            uint32_t slot = atomicAdd(n_out, 1u);
            qout[slot] = make_uint2(refs[c], child_base + int_rank);
            ++int_rank;
        }
        meta[s >> 2] |= m << (8 * (s & 3));
    }
    Node8 nd;
    quantize_node(nlo, nhi, slo, shi, used, imask, nd, err);
    nd.b = make_uint4(child_base, tri_base, meta[0], meta[1]);
    nodes[q.y] = nd;
}

template <typename T>
cudaError_t dalloc(T** p, size_t count) {
    return cudaMalloc((void**)p, sizeof(T) * (count ? count : 1));
}

}  // namespace

cudaError_t build_bvh8(const BvhInputs& in, cudaStream_t st, BvhOutputs* out, std::string* msg) {
    uint32_t n = in.n_tris;
    out->nodes = nullptr;
    out->tris = nullptr;
    out->tri_inst = nullptr;
    out->n_nodes = 0;
    out->depth = 0;
    out->kernel_launches = 0;
    cudaError_t e = cudaSuccess;
#define CK(x)                                         \
    do {                                              \
        e = (x);                                      \
        if (e != cudaSuccess) {                       \
            if (msg) *msg = std::string(#x) + ": " + cudaGetErrorString(e); \
            goto done;                                \
        }                                             \
    } while (0)
    TriSlot* flat = nullptr;
    float4* cen = nullptr;
    uint32_t *bounds = nullptr, *keys = nullptr, *vals = nullptr, *keys2 = nullptr, *vals2 = nullptr,
             *scratch = nullptr, *counters = nullptr, *err = nullptr;
    uint2 *qa = nullptr, *qb = nullptr;
    SahTask* sah_tasks[2] = {nullptr, nullptr};
    uint32_t* sah_bins = nullptr;
    Bvh2 b{};
    if (n == 0) return cudaSuccess;
    {
        CK(dalloc(&out->tri_inst, n));
        CK(dalloc(&out->tris, n));
        uint32_t node_cap = n > 1 ? n - 1 : 1;
        CK(dalloc(&out->nodes, node_cap));
        CK(dalloc(&flat, n));
        CK(dalloc(&cen, n));
        CK(dalloc(&bounds, 6));
        CK(dalloc(&keys, n));
        CK(dalloc(&vals, n));
        CK(dalloc(&keys2, n));
        CK(dalloc(&vals2, n));
        CK(dalloc(&scratch, radix_scratch_words(n)));
        CK(dalloc(&counters, 4));
        CK(dalloc(&err, 1));
        CK(dalloc(&qa, node_cap));
        CK(dalloc(&qb, node_cap));
        CK(dalloc(&b.inode, node_cap));
        CK(dalloc(&b.ibox, 2 * (size_t)node_cap));
        CK(dalloc(&b.lbox, 2 * (size_t)n));
        CK(dalloc(&b.iparent, node_cap));
        CK(dalloc(&b.lparent, n));
        CK(dalloc(&b.flags, node_cap));
        uint32_t init_bounds[6] = {0xFFFFFFFFu, 0xFFFFFFFFu, 0xFFFFFFFFu, 0u, 0u, 0u};
        CK(cudaMemcpyAsync(bounds, init_bounds, sizeof(init_bounds), cudaMemcpyHostToDevice, st));
        CK(cudaMemsetAsync(b.flags, 0, sizeof(uint32_t) * node_cap, st));
        CK(cudaMemsetAsync(err, 0, 4, st));
        const int B = 256;
        uint32_t grid = (n + B - 1) / B;
        k_flatten<<<grid, B, 0, st>>>(in.vtx, in.indices, in.mesh_infos, in.inst, in.fwd, in.n_inst, n, flat,
                                      out->tri_inst, cen, bounds);
        ++out->kernel_launches;
        uint32_t* sv = nullptr;
        if (in.builder == BVH_BUILDER_LBVH || n < 2) {
            k_morton<<<grid, B, 0, st>>>(cen, bounds, n, keys, vals);
            ++out->kernel_launches;
            uint32_t* sk;
            out->kernel_launches += sort_pairs(keys, vals, keys2, vals2, n, nullptr, 0, 30, scratch, st, &sk, &sv);
            if (n > 1) {
                k_karras<<<(n - 1 + B - 1) / B, B, 0, st>>>(sk, (int)n, b);
                ++out->kernel_launches;
            }
        } else {
            // binned SAH, level by level (keys/vals/keys2/vals2 serve as the
            // permutation and position -> task ping-pong buffers)
            uint32_t *perm = keys, *perm2 = keys2;
            int *pt = (int*)vals, *pt2 = (int*)vals2;
            const uint32_t task_cap = n / 2 + 1;
            // tasks that bin in global memory hold more than SAH_SMALL primitives
            // of disjoint ranges: at most n / (SAH_SMALL + 1) per level
            const uint32_t bin_cap = n / (SAH_SMALL + 1) + 1;
            CK(dalloc(&sah_tasks[0], task_cap));
            CK(dalloc(&sah_tasks[1], task_cap));
            CK(dalloc(&sah_bins, (size_t)bin_cap * SAH_TASK_WORDS));
            // counters: node alloc, -, next tasks, bin slots of the next level
            CK(cudaMemcpyAsync(counters, std::array<uint32_t, 4>{1u, 0u, 0u, 0u}.data(), 16, cudaMemcpyHostToDevice, st));
            k_sah_root<<<grid, B, 0, st>>>(bounds, n, sah_tasks[0], pt, perm, counters + 3, bin_cap);
            ++out->kernel_launches;
            uint32_t n_tasks = 1, n_bins = 1, level = 0;
            while (n_tasks > 0) {
                uint32_t words = n_bins * SAH_TASK_WORDS;
                if (words) k_sah_init_bins<<<(words + 255) / 256, 256, 0, st>>>(sah_bins, words);
                k_sah_bin<<<grid, B, 0, st>>>(perm, pt, n, sah_tasks[0], cen, flat, sah_bins);
                CK(cudaMemsetAsync(counters + 2, 0, 8, st));
                k_sah_split<<<(n_tasks + 127) / 128, 128, 0, st>>>(sah_tasks[0], n_tasks, sah_bins, perm, cen, flat,
                                                                   sah_tasks[1],
                                                                   counters + 2, task_cap, counters + 3, bin_cap,
                                                                   counters, n - 1, b, level, err);
                k_sah_partition<<<grid, B, 0, st>>>(perm, pt, n, sah_tasks[0], cen, perm2, pt2);
                out->kernel_launches += 4;
                CK(cudaGetLastError());
                uint32_t hc2[2];
                CK(cudaMemcpyAsync(hc2, counters + 2, 8, cudaMemcpyDeviceToHost, st));
                CK(cudaStreamSynchronize(st));
                n_tasks = hc2[0];
                n_bins = std::min(hc2[1], bin_cap);
                std::swap(perm, perm2);
                std::swap(pt, pt2);
                std::swap(sah_tasks[0], sah_tasks[1]);
                if (n_tasks > task_cap || ++level > 4096) {
                    if (msg) *msg = "binned SAH build did not converge";
                    e = cudaErrorUnknown;
                    goto done;
                }
            }
            sv = perm;
        }
        k_refit<<<grid, B, 0, st>>>(flat, sv, (int)n, b);
        ++out->kernel_launches;
        CK(cudaGetLastError());
        // collapse, level by level; node 0 is the root
        uint2 root = make_uint2(n > 1 ? 0u : LEAF, 0u);
        uint32_t init_counts[4] = {1u, 0u, 0u, 0u};  // node alloc, tri alloc, queue out count, pad
        CK(cudaMemcpyAsync(qa, &root, sizeof(root), cudaMemcpyHostToDevice, st));
        CK(cudaMemcpyAsync(counters, init_counts, sizeof(init_counts), cudaMemcpyHostToDevice, st));
        uint32_t n_in = 1;
        uint32_t depth = 0;
        out->level_start[0] = 0u;
        out->level_start[1] = 1u;
        while (n_in > 0) {
            CK(cudaMemsetAsync(counters + 2, 0, 4, st));
            k_collapse<<<(n_in + 127) / 128, 128, 0, st>>>(b, qa, n_in, qb, counters + 2, out->nodes, counters,
                                                           node_cap, out->tris, counters + 1, n, flat, sv, err,
                                                           in.width < 2 ? 2 : (in.width > 8 ? 8 : in.width),
                                                           in.leaf_max < 1u ? 1u : (in.leaf_max > LEAF_MAX_LIMIT ? LEAF_MAX_LIMIT : in.leaf_max));
            ++out->kernel_launches;
            ++depth;
            CK(cudaGetLastError());
            uint32_t hc3[3];
            CK(cudaMemcpyAsync(hc3, counters, sizeof(hc3), cudaMemcpyDeviceToHost, st));
            CK(cudaStreamSynchronize(st));
            n_in = hc3[2];
            if (depth < 65) out->level_start[depth + 1] = hc3[0];  // nodes of the next level end here
            uint2* t = qa;
            qa = qb;
            qb = t;
            if (depth > 64) {
                if (msg) *msg = "BVH8 collapse exceeded 64 levels";
                e = cudaErrorUnknown;
                goto done;
            }
        }
        uint32_t hc[4], herr = 0;
        CK(cudaMemcpyAsync(hc, counters, sizeof(hc), cudaMemcpyDeviceToHost, st));
        CK(cudaMemcpyAsync(&herr, err, 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
        if (herr != 0u || hc[1] != n) {
            if (msg) *msg = "BVH8 collapse produced an inconsistent tree";
            e = cudaErrorUnknown;
            goto done;
        }
        out->n_nodes = hc[0];
        out->depth = depth;
    }
done:
    cudaFree(sah_tasks[0]);
    cudaFree(sah_tasks[1]);
    cudaFree(sah_bins);
    cudaFree(flat);
    cudaFree(cen);
    cudaFree(bounds);
    cudaFree(keys);
    cudaFree(vals);
    cudaFree(keys2);
    cudaFree(vals2);
    cudaFree(scratch);
    cudaFree(counters);
    cudaFree(err);
    cudaFree(qa);
    cudaFree(qb);
    cudaFree(b.inode);
    cudaFree(b.ibox);
    cudaFree(b.lbox);
    cudaFree(b.iparent);
    cudaFree(b.lparent);
    cudaFree(b.flags);
    if (e != cudaSuccess) {
        cudaFree(out->nodes);
        cudaFree(out->tris);
        cudaFree(out->tri_inst);
        out->nodes = nullptr;
        out->tris = nullptr;
        out->tri_inst = nullptr;
    }
#undef CK
    return e;
}

int launch_update_slots(TriSlot* tris, uint32_t n_tris, const uint32_t* tri_inst, const uint8_t* moved,
                        const float4* vtx, const uint32_t* indices, const uint4* mesh_infos, const InstDev* inst,
                        const InstFwd* fwd, cudaStream_t st) {
    if (n_tris == 0) return 0;
    k_update_slots<<<(n_tris + 255) / 256, 256, 0, st>>>(tris, n_tris, tri_inst, moved, vtx, indices, mesh_infos, inst,
                                                         fwd);
    return 1;
}

int launch_expand_lights(const LightInst* li, uint32_t n_li, const uint8_t* moved, const float4* vtx,
                         const uint32_t* indices, const uint4* mesh_infos, const InstDev* inst, const InstFwd* fwd,
                         float4* lights, cudaStream_t st) {
    if (n_li == 0) return 0;
    k_expand_lights<<<n_li, 128, 0, st>>>(li, moved, vtx, indices, mesh_infos, inst, fwd, lights);
    return 1;
}

int refit_bvh8(Node8* nodes, const TriSlot* tris, const BvhOutputs& lv, float4* aux, uint32_t* err,
               cudaStream_t st) {
    int n = 0;
    for (int L = (int)lv.depth - 1; L >= 0; --L) {
        uint32_t b = lv.level_start[L], e = lv.level_start[L + 1];
        if (e <= b) continue;
        k_refit8<<<(e - b + 127) / 128, 128, 0, st>>>(nodes, tris, b, e, aux, err);
        ++n;
    }
    return n;
}

}  // namespace srt

// bvh_build.h — interface of the GPU BVH8 builder (bvh_build.cu).
#pragma once

#include <string>

#include "device_common.cuh"

namespace srt {

// Rows of an instance's object-to-world 3x4 affine transform.
struct InstFwd {
    float4 r0, r1, r2;
};

// Object -> world with every rounding pinned (((m0 x + m1 y) + m2 z) + m3),
// the order of the host builder's light expansion, so the flattened
// triangles, the refit and the light expansion agree bit for bit.
__device__ __forceinline__ float3 xform_point(const InstFwd& f, float x, float y, float z) {
    return make_float3(
        __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(f.r0.x, x), __fmul_rn(f.r0.y, y)), __fmul_rn(f.r0.z, z)), f.r0.w),
        __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(f.r1.x, x), __fmul_rn(f.r1.y, y)), __fmul_rn(f.r1.z, z)), f.r1.w),
        __fadd_rn(__fadd_rn(__fadd_rn(__fmul_rn(f.r2.x, x), __fmul_rn(f.r2.y, y)), __fmul_rn(f.r2.z, z)), f.r2.w));
}

// A light instance (add_light_instance): its triangles' world-space copies
// are lights[first .. first + count).
struct LightInst {
    uint32_t inst, first, count, pad;
    float4 params;
};

constexpr int BVH_BUILDER_SAH = 0;   // binned SAH, top-down (default)
constexpr int BVH_BUILDER_LBVH = 1;  // Morton-ordered LBVH (Karras 2012)

struct BvhInputs {
    const float4* vtx;        // device srt_vertex array (pos, normal)
    const uint32_t* indices;  // device global index buffer
    const uint4* mesh_infos;  // device srt_mesh_info array
    const InstDev* inst;      // device, sorted by tri_offset
    const InstFwd* fwd;       // device, one per instance
    uint32_t n_inst;
    uint32_t n_tris;          // flattened triangle count
    int builder;              // BVH_BUILDER_*
    int width = 8;            // children per node, 2..8 (nodes keep the 8-slot format)
    uint32_t leaf_max = 2;    // triangles of the largest leaf, 1..3 (8 leaves share 24 triangle bits)
};

struct BvhOutputs {
    Node8* nodes;        // device, n_nodes entries (node 0 = root)
    TriSlot* tris;       // device, n_tris leaf slots
    uint32_t* tri_inst;  // device, flattened triangle -> instance
    uint32_t n_nodes;
    uint32_t depth;      // number of 8-wide levels
    int kernel_launches;
    uint32_t level_start[66];  // nodes of level L: [level_start[L], level_start[L + 1]), L < depth
};

// Builds the tree on `st` (synchronising it); device memory in `out` is
// owned by the caller afterwards (cudaFree).
cudaError_t build_bvh8(const BvhInputs& in, cudaStream_t st, BvhOutputs* out, std::string* msg);

// Scene updates (moved instances), all on `st`:
// re-transform the leaf slots of instances with moved[inst] != 0,
int launch_update_slots(TriSlot* tris, uint32_t n_tris, const uint32_t* tri_inst, const uint8_t* moved,
                        const float4* vtx, const uint32_t* indices, const uint4* mesh_infos, const InstDev* inst,
                        const InstFwd* fwd, cudaStream_t st);
// expand light instances (all, or those with moved[inst] != 0) into world-space lights,
int launch_expand_lights(const LightInst* li, uint32_t n_li, const uint8_t* moved, const float4* vtx,
                         const uint32_t* indices, const uint4* mesh_infos, const InstDev* inst, const InstFwd* fwd,
                         float4* lights, cudaStream_t st);
// recompute every node's boxes bottom-up (topology kept) and re-quantise;
// aux: 2 float4 per node of scratch; err: device error word.
int refit_bvh8(Node8* nodes, const TriSlot* tris, const BvhOutputs& levels, float4* aux, uint32_t* err,
               cudaStream_t st);

}  // namespace srt

// bvh_build.h — interface of the GPU BVH8 builder (bvh_build.cu).
#pragma once

#include <string>

#include "device_common.cuh"

namespace srt {

// Rows of an instance's object-to-world 3x4 affine transform.
struct InstFwd {
    float4 r0, r1, r2;
};

struct BvhInputs {
    const float4* vtx;        // device srt_vertex array (pos, normal)
    const uint32_t* indices;  // device global index buffer
    const uint4* mesh_infos;  // device srt_mesh_info array
    const InstDev* inst;      // device, sorted by tri_offset
    const InstFwd* fwd;       // device, one per instance
    uint32_t n_inst;
    uint32_t n_tris;          // flattened triangle count
};

struct BvhOutputs {
    Node8* nodes;        // device, n_nodes entries (node 0 = root)
    TriSlot* tris;       // device, n_tris leaf slots
    uint32_t* tri_inst;  // device, flattened triangle -> instance
    uint32_t n_nodes;
    uint32_t depth;      // number of 8-wide levels
    int kernel_launches;
};

// Builds the tree on `st` (synchronising it); device memory in `out` is
// owned by the caller afterwards (cudaFree).
cudaError_t build_bvh8(const BvhInputs& in, cudaStream_t st, BvhOutputs* out, std::string* msg);

}  // namespace srt

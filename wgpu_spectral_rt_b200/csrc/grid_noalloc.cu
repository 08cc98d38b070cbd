// grid_noalloc.cu — photon hash grid over a device-resident photon set that
// performs no device allocation at all.
//
// Some callers cannot call cudaMalloc: an engine or framework whose own pool
// allocator already owns the device memory (a raw cudaMalloc behind its back
// can fail or fragment that pool), or a real-time frame loop that forbids any
// allocation once it has started.  For them this entry point takes its
// temporary storage from one file-scope __device__ array of fixed size, and
// works only on buffers the caller already owns.
//
// The array (GRID_NOALLOC_SCRATCH_WORDS 32-bit words, 16.5 MiB) lives in
// every GPU that loads this library until the process exits.  Every call
// shares it, so calls that overlap on the GPU (concurrent streams, or several
// host threads) race on it and must be serialised by the caller.  Each call
// writes every scratch word it later reads, so the contents left by the
// previous call never leak into a result.
#include <mutex>

#include "radix_sort.cuh"
#include "render_kernels.h"

namespace srt {

// Photon capacity of the scratch: the reference's MAX_PHOTONS (2^20).
constexpr uint32_t GRID_NOALLOC_MAX_PHOTONS = 1u << 20;
// keys, values and their ping-pong copies (4 words per photon) + sort histograms
constexpr size_t GRID_NOALLOC_SCRATCH_WORDS =
    4ull * GRID_NOALLOC_MAX_PHOTONS + 256ull * (GRID_NOALLOC_MAX_PHOTONS / RS_TILE) + 256ull;

static __device__ __align__(256) uint32_t g_grid_noalloc_scratch[GRID_NOALLOC_SCRATCH_WORDS];

namespace {

__global__ void k_noalloc_keys(const float4* __restrict__ photons, uint32_t n, uint32_t frame, float cell,
                               uint32_t hash_bits, uint32_t* __restrict__ keys, uint32_t* __restrict__ vals) {
    float3 j = grid_jitter(frame, cell);
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        float4 p0 = photons[2 * i], p1 = photons[2 * i + 1];
        keys[i] = p1.w == 0.0f ? (1u << hash_bits) : grid_hash(xyz(p0), j, cell, hash_bits);
        vals[i] = i;
    }
}

// Sorted (hash, index) pairs -> 64-bit keys and the [start, end) range of
// every non-empty bucket (ranges were cleared before).
__global__ void k_noalloc_ranges(const uint32_t* __restrict__ keys, const uint32_t* __restrict__ vals, uint32_t n,
                                 uint32_t hash_bits, unsigned long long* __restrict__ keys_out,
                                 uint2* __restrict__ ranges) {
    uint32_t sentinel = 1u << hash_bits;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        uint32_t h = keys[i];
        if (keys_out) keys_out[i] = ((unsigned long long)h << 32) | vals[i];
        if (ranges == nullptr || h >= sentinel) continue;
        if (i == 0 || keys[i - 1] != h) ranges[h].x = i;
        if (i + 1 == n || keys[i + 1] != h) ranges[h].y = i + 1;
    }
}

std::mutex g_mu;
uint32_t* g_scratch_ptr[64] = {};  // device address of the scratch array, per device ordinal

}  // namespace

}  // namespace srt

using namespace srt;

extern "C" srt_status srt_photon_grid_build_noalloc(void* stream, const srt_photon* photons, uint32_t n,
                                                    uint32_t frame_count, float cell_size, uint32_t hash_bits,
                                                    uint64_t* keys_out, uint32_t* ranges_out) {
    std::lock_guard<std::mutex> lock(g_mu);
    static_assert(GRID_NOALLOC_MAX_PHOTONS == SRT_GRID_NOALLOC_MAX_PHOTONS, "header and scratch disagree");
    if (n > GRID_NOALLOC_MAX_PHOTONS) return SRT_ERR_CAPACITY;
    if ((n && !photons) || hash_bits < 4 || hash_bits > 26 || !(cell_size > 0.f)) return SRT_ERR_INVALID_ARG;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= 64) return SRT_ERR_CUDA;
    if (!g_scratch_ptr[dev]) {
        // first call on this device (with it current): host code may not use
        // the array's name as an address, so look the device address up once
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_grid_noalloc_scratch);
        if (e != cudaSuccess || !p) return SRT_ERR_CUDA;
        g_scratch_ptr[dev] = (uint32_t*)p;
    }
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* s = g_scratch_ptr[dev];
    uint32_t* keys = s;
    uint32_t* vals = s + GRID_NOALLOC_MAX_PHOTONS;
    uint32_t* keys2 = s + 2ull * GRID_NOALLOC_MAX_PHOTONS;
    uint32_t* vals2 = s + 3ull * GRID_NOALLOC_MAX_PHOTONS;
    uint32_t* hist = s + 4ull * GRID_NOALLOC_MAX_PHOTONS;
    if (ranges_out) {
        e = cudaMemsetAsync(ranges_out, 0, sizeof(uint2) << hash_bits, st);
        if (e != cudaSuccess) return SRT_ERR_CUDA;
    }
    if (n > 0) {
        const uint32_t grid = 148 * 8;
        k_noalloc_keys<<<grid, 256, 0, st>>>(reinterpret_cast<const float4*>(photons), n, frame_count, cell_size,
                                             hash_bits, keys, vals);
        uint32_t *sk, *sv;
        sort_pairs(keys, vals, keys2, vals2, n, nullptr, 0, (int)hash_bits + 1, hist, st, &sk, &sv);
        k_noalloc_ranges<<<grid, 256, 0, st>>>(sk, sv, n, hash_bits, reinterpret_cast<unsigned long long*>(keys_out),
                                               reinterpret_cast<uint2*>(ranges_out));
    }
    return cudaGetLastError() == cudaSuccess ? SRT_OK : SRT_ERR_CUDA;
}

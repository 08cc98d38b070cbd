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
#include <cstdint>
#include <mutex>
#include <utility>

#include <cuda.h>

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

// The scratch array's device address belongs to the CUDA context that was
// current when it was looked up.  It is cached per device ordinal together
// with that context's unique id (cuCtxGetId), and looked up again when the
// current context is a different one (after cudaDeviceReset, or a context
// the caller made current through the driver API).  The driver entry points
// are resolved through the runtime, so the library does not link libcuda.
struct ScratchAddr {
    unsigned long long ctx_id;
    uint32_t* ptr;
};
ScratchAddr g_scratch[64] = {};

typedef CUresult (*PfnCtxGetCurrent)(CUcontext*);
typedef CUresult (*PfnCtxGetId)(CUcontext, unsigned long long*);

// Unique id of the calling thread's current context; 0 when none is current
// yet or the driver does not report ids.
unsigned long long current_ctx_id() {
    static PfnCtxGetCurrent get_current = nullptr;
    static PfnCtxGetId get_id = nullptr;
    static bool resolved = false;
    if (!resolved) {
        resolved = true;
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_current = (PfnCtxGetCurrent)f;
        f = nullptr;
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            get_id = (PfnCtxGetId)f;
        (void)cudaGetLastError();  // a failed lookup leaves nothing pending
    }
    if (!get_current || !get_id) return 0;
    CUcontext c = nullptr;
    if (get_current(&c) != CUDA_SUCCESS || !c) return 0;
    unsigned long long id = 0;
    return get_id(c, &id) == CUDA_SUCCESS ? id : 0;
}

// Launches with the status of this launch alone: cudaLaunchKernelEx returns
// it directly, so an error that an earlier, unrelated call left pending on
// this thread is neither reported as ours nor cleared.
template <typename... P, typename... A>
cudaError_t launch(void (*k)(P...), uint32_t grid, uint32_t block, cudaStream_t st, A&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaError_t e = cudaLaunchKernelEx(&cfg, k, std::forward<A>(args)...);
    if (e != cudaSuccess) (void)cudaGetLastError();  // the pending error is this launch's own
    return e;
}

// sort_pairs (radix_sort.cuh) with every launch checked as above.
cudaError_t sort_pairs_checked(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt, uint32_t n,
                               int end_bit, uint32_t* scratch, cudaStream_t st, uint32_t** out_keys,
                               uint32_t** out_vals) {
    const uint32_t tiles = (n + RS_TILE - 1) / RS_TILE;
    uint32_t* hist = scratch;
    uint32_t* row_total = scratch + (size_t)256 * tiles;
    const uint32_t* no_dev_count = nullptr;
    uint32_t *ki = keys, *vi = vals, *ko = keys_alt, *vo = vals_alt;
    for (int shift = 0; shift < end_bit; shift += 8) {
        cudaError_t e = launch(k_rs_upsweep, tiles, RS_THREADS, st, (const uint32_t*)ki, no_dev_count, n, shift,
                               tiles, hist);
        if (e == cudaSuccess) e = launch(k_rs_rowscan, 256u, 1024u, st, hist, tiles, row_total);
        if (e == cudaSuccess)
            e = launch(k_rs_scatter, tiles, RS_THREADS, st, (const uint32_t*)ki, (const uint32_t*)vi, ko, vo,
                       no_dev_count, n, shift, tiles, (const uint32_t*)hist, (const uint32_t*)row_total);
        if (e != cudaSuccess) return e;
        uint32_t* t = ki;
        ki = ko;
        ko = t;
        t = vi;
        vi = vo;
        vo = t;
    }
    *out_keys = ki;
    *out_vals = vi;
    return cudaSuccess;
}

}  // namespace

}  // namespace srt

using namespace srt;

extern "C" srt_status srt_photon_grid_build_noalloc(void* stream, const srt_photon* photons, uint32_t n,
                                                    uint32_t frame_count, float cell_size, uint32_t hash_bits,
                                                    uint64_t* keys_out, uint32_t* ranges_out) {
    static_assert(GRID_NOALLOC_MAX_PHOTONS == SRT_GRID_NOALLOC_MAX_PHOTONS, "header and scratch disagree");
    if (n > GRID_NOALLOC_MAX_PHOTONS) return SRT_ERR_CAPACITY;
    if ((n && !photons) || hash_bits < 4 || hash_bits > 26 || !(cell_size > 0.f)) return SRT_ERR_INVALID_ARG;
    // photons are read as float4 pairs, keys written as u64 and ranges as
    // uint2: refuse misaligned pointers before any device work
    if (((uintptr_t)photons & 15u) || ((uintptr_t)keys_out & 7u) || ((uintptr_t)ranges_out & 7u))
        return SRT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lock(g_mu);
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) {
        (void)cudaGetLastError();
        return e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver ? SRT_ERR_NO_DEVICE : SRT_ERR_CUDA;
    }
    if (dev < 0 || dev >= 64) return SRT_ERR_CUDA;
    unsigned long long ctx = current_ctx_id();
    ScratchAddr& sa = g_scratch[dev];
    if (!sa.ptr || (ctx != 0 && ctx != sa.ctx_id)) {
        // set-up, with this device current: host code may not use the
        // array's name as an address, so look its device address up (once
        // per device and context; cudaGetSymbolAddress allocates nothing)
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_grid_noalloc_scratch);
        if (e != cudaSuccess || !p) {
            (void)cudaGetLastError();
            return SRT_ERR_CUDA;
        }
        sa.ptr = (uint32_t*)p;
        sa.ctx_id = ctx != 0 ? ctx : current_ctx_id();  // the lookup made the primary context current
    }
    cudaStream_t st = (cudaStream_t)stream;
    uint32_t* s = sa.ptr;
    uint32_t* keys = s;
    uint32_t* vals = s + GRID_NOALLOC_MAX_PHOTONS;
    uint32_t* keys2 = s + 2ull * GRID_NOALLOC_MAX_PHOTONS;
    uint32_t* vals2 = s + 3ull * GRID_NOALLOC_MAX_PHOTONS;
    uint32_t* hist = s + 4ull * GRID_NOALLOC_MAX_PHOTONS;
    if (ranges_out) {
        e = cudaMemsetAsync(ranges_out, 0, sizeof(uint2) << hash_bits, st);
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            return SRT_ERR_CUDA;
        }
    }
    if (n == 0) return SRT_OK;
    const uint32_t grid = 148 * 8;
    e = launch(k_noalloc_keys, grid, 256u, st, reinterpret_cast<const float4*>(photons), n, frame_count, cell_size,
               hash_bits, keys, vals);
    uint32_t *sk = nullptr, *sv = nullptr;
    if (e == cudaSuccess) e = sort_pairs_checked(keys, vals, keys2, vals2, n, (int)hash_bits + 1, hist, st, &sk, &sv);
    if (e == cudaSuccess)
        e = launch(k_noalloc_ranges, grid, 256u, st, (const uint32_t*)sk, (const uint32_t*)sv, n, hash_bits,
                   reinterpret_cast<unsigned long long*>(keys_out), reinterpret_cast<uint2*>(ranges_out));
    return e == cudaSuccess ? SRT_OK : SRT_ERR_CUDA;
}

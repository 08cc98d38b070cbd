// radix_sort.cuh — stable LSD radix sort of (u32 key, u32 value) pairs.
//
// Three kernels per 8-bit digit pass:
//   upsweep  per-tile digit histogram, stored digit-major hist[d * tiles + t]
//   rowscan  one block per digit: exclusive scan of its row, row total
//   scatter  per tile: stable rank of every item among equal digits of the
//            tile (warp match_any per 32-item round, per-warp counters in
//            shared memory), plus the tile's global digit offset
// The element count may live in device memory (n_dev), so the same launches
// serve a count produced on the GPU and can be captured in a CUDA graph;
// tiles at or beyond the count exit after zeroing their histogram column.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace srt {

constexpr int RS_WARPS = 8;
constexpr int RS_THREADS = RS_WARPS * 32;
constexpr int RS_IPT = 8;                        // items per thread per tile
constexpr int RS_TILE = RS_THREADS * RS_IPT;     // 2048 items

__device__ __forceinline__ uint32_t rs_count(const uint32_t* n_dev, uint32_t n_host) {
    return n_dev ? *n_dev : n_host;
}

static __global__ void __launch_bounds__(RS_THREADS) k_rs_upsweep(const uint32_t* __restrict__ keys, const uint32_t* n_dev,
                                                            uint32_t n_host, int shift, uint32_t tiles,
                                                            uint32_t* __restrict__ hist) {
    __shared__ uint32_t h[256];
    uint32_t t = blockIdx.x;
    h[threadIdx.x] = 0u;
    __syncthreads();
    uint32_t n = rs_count(n_dev, n_host);
    uint64_t base = (uint64_t)t * RS_TILE;
    if (base < n) {
        uint32_t end = (uint32_t)((uint64_t)n < base + RS_TILE ? (uint64_t)n : base + RS_TILE);
        for (uint32_t i = (uint32_t)base + threadIdx.x; i < end; i += RS_THREADS)
            atomicAdd(&h[(keys[i] >> shift) & 0xFFu], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * tiles + t] = h[threadIdx.x];
}

// One block (1024 threads) per digit row; rows hold `tiles` counters.
static __global__ void __launch_bounds__(1024) k_rs_rowscan(uint32_t* __restrict__ hist, uint32_t tiles,
                                                      uint32_t* __restrict__ row_total) {
    __shared__ uint32_t warp_sums[32];
    __shared__ uint32_t carry;
    uint32_t* row = hist + (size_t)blockIdx.x * tiles;
    if (threadIdx.x == 0) carry = 0u;
    __syncthreads();
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (uint32_t base = 0; base < tiles; base += 1024) {
        uint32_t i = base + threadIdx.x;
        uint32_t v = i < tiles ? row[i] : 0u;
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) warp_sums[warp] = x;
        __syncthreads();
        if (warp == 0) {
            uint32_t s = warp_sums[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                uint32_t y = __shfl_up_sync(0xFFFFFFFFu, s, o);
                if (lane >= o) s += y;
            }
            warp_sums[lane] = s;
        }
        __syncthreads();
        uint32_t excl = carry + (warp ? warp_sums[warp - 1] : 0u) + x - v;
        if (i < tiles) row[i] = excl;
        __syncthreads();
        if (threadIdx.x == 1023) carry = excl + v;
        __syncthreads();
    }
    if (threadIdx.x == 0) row_total[blockIdx.x] = carry;
}

static __global__ void __launch_bounds__(RS_THREADS) k_rs_scatter(const uint32_t* __restrict__ keys_in,
                                                            const uint32_t* __restrict__ vals_in,
                                                            uint32_t* __restrict__ keys_out,
                                                            uint32_t* __restrict__ vals_out, const uint32_t* n_dev,
                                                            uint32_t n_host, int shift, uint32_t tiles,
                                                            const uint32_t* __restrict__ hist,
                                                            const uint32_t* __restrict__ row_total) {
    __shared__ uint32_t cnt[RS_WARPS][256];
    __shared__ uint32_t digit_base[256];
    uint32_t n = rs_count(n_dev, n_host);
    uint64_t tile_base = (uint64_t)blockIdx.x * RS_TILE;
    if (tile_base >= n) return;
    int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int d = threadIdx.x; d < RS_WARPS * 256; d += RS_THREADS) (&cnt[0][0])[d] = 0u;
    // digit base = exclusive scan of row totals (256 entries, one per thread)
    {
        uint32_t v = row_total[threadIdx.x];
        uint32_t x = v;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xFFFFFFFFu, x, o);
            if (lane >= o) x += y;
        }
        __shared__ uint32_t ws[RS_WARPS];
        if (lane == 31) ws[warp] = x;
        __syncthreads();
        uint32_t add = 0;
        for (int w = 0; w < warp; ++w) add += ws[w];
        digit_base[threadIdx.x] = add + x - v + hist[threadIdx.x * tiles + blockIdx.x];
    }
    __syncthreads();
    uint32_t k[RS_IPT], val[RS_IPT], rank[RS_IPT];
    uint64_t warp_base = tile_base + (uint64_t)warp * 32 * RS_IPT;
    uint32_t lt = (1u << lane) - 1u;
#pragma unroll
    for (int r = 0; r < RS_IPT; ++r) {
        uint64_t i = warp_base + (uint64_t)r * 32 + lane;
        bool valid = i < n;
        k[r] = valid ? keys_in[i] : 0u;
        val[r] = valid ? vals_in[i] : 0u;
        uint32_t d = (k[r] >> shift) & 0xFFu;
        uint32_t act = __ballot_sync(0xFFFFFFFFu, valid);
        uint32_t peers = __match_any_sync(0xFFFFFFFFu, valid ? d : 0x100u);
        peers &= act;
        uint32_t before = valid ? cnt[warp][d] : 0u;
        rank[r] = before + __popc(peers & lt);
        __syncwarp();
        if (valid && (peers & lt) == 0u) cnt[warp][d] = before + __popc(peers);
        __syncwarp();
    }
    __syncthreads();
    // exclusive prefix over warps, one digit per thread
    {
        uint32_t run = 0;
        for (int w = 0; w < RS_WARPS; ++w) {
            uint32_t c = cnt[w][threadIdx.x];
            cnt[w][threadIdx.x] = run;
            run += c;
        }
    }
    __syncthreads();
#pragma unroll
    for (int r = 0; r < RS_IPT; ++r) {
        uint64_t i = warp_base + (uint64_t)r * 32 + lane;
        if (i < n) {
            uint32_t d = (k[r] >> shift) & 0xFFu;
            uint32_t pos = digit_base[d] + cnt[warp][d] + rank[r];
            keys_out[pos] = k[r];
            vals_out[pos] = val[r];
        }
    }
}

// Scratch for sort_pairs: 256 * tiles + 256 counters.
inline size_t radix_scratch_words(uint32_t max_n) {
    uint32_t tiles = (max_n + RS_TILE - 1) / RS_TILE;
    if (tiles == 0) tiles = 1;
    return (size_t)256 * tiles + 256;
}

// Sorts bits [begin_bit, end_bit) of (keys, vals), ping-ponging with the
// alternate buffers; *out_keys / *out_vals receive whichever pair holds the
// result.  max_n bounds the count for the launch grid; n_dev (optional)
// holds the actual count.  Returns the number of kernels launched.
inline int sort_pairs(uint32_t* keys, uint32_t* vals, uint32_t* keys_alt, uint32_t* vals_alt, uint32_t max_n,
                      const uint32_t* n_dev, int begin_bit, int end_bit, uint32_t* scratch, cudaStream_t st,
                      uint32_t** out_keys, uint32_t** out_vals) {
    uint32_t tiles = (max_n + RS_TILE - 1) / RS_TILE;
    uint32_t *ki = keys, *vi = vals, *ko = keys_alt, *vo = vals_alt;
    int launches = 0;
    if (tiles > 0) {
        uint32_t* hist = scratch;
        uint32_t* row_total = scratch + (size_t)256 * tiles;
        for (int shift = begin_bit; shift < end_bit; shift += 8) {
            k_rs_upsweep<<<tiles, RS_THREADS, 0, st>>>(ki, n_dev, max_n, shift, tiles, hist);
            k_rs_rowscan<<<256, 1024, 0, st>>>(hist, tiles, row_total);
            k_rs_scatter<<<tiles, RS_THREADS, 0, st>>>(ki, vi, ko, vo, n_dev, max_n, shift, tiles, hist, row_total);
            launches += 3;
            uint32_t* t = ki;
            ki = ko;
            ko = t;
            t = vi;
            vi = vo;
            vo = t;
        }
    }
    *out_keys = ki;
    *out_vals = vi;
    return launches;
}

}  // namespace srt

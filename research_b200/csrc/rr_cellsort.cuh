// rr_cellsort.cuh — the grid guide's sample grouping: a stable sort of
// sample indices by cell (least-significant-digit radix sort, 8-bit digits)
// and an exclusive scan, hand-written for one GPU.
//
// A pass over digit (key >> shift) & 255:
//   sort_hist_kernel    each tile of kSortTile consecutive items counts its
//                       digits; counts are stored digit-major, tile-minor
//   scan_exclusive      turns those counts into the first output position
//                       of every (digit, tile)
//   sort_scatter_kernel each tile writes its items there, in index order
//                       within a digit: warp w owns the tile's items
//                       [w*256, w*256+256) in eight 32-item chunks, so per
//                       digit the tile's earlier warps, then the warp's
//                       earlier chunks, then its lower lanes come first
// Every pass is stable, so after ceil(key bits / 8) passes the items are
// ordered by key and, within a key, by index; the result does not depend on
// timing (no atomics decide an order).
#pragma once

#include <cstdint>

namespace rr {

constexpr int kSortThreads = 256;                       // one digit per thread in the histogram
constexpr int kSortItems = 8;
constexpr int kSortTile = kSortThreads * kSortItems;    // items per tile
constexpr int kSortBins = 256;
constexpr int kSortWarps = kSortThreads / 32;
static_assert(kSortThreads == kSortBins && kSortTile == kSortWarps * 32 * kSortItems, "tile shape");

__global__ void __launch_bounds__(kSortThreads) sort_hist_kernel(const uint32_t* __restrict__ keys, uint32_t n,
                                                                 int shift, uint32_t tiles,
                                                                 uint32_t* __restrict__ hist) {
    __shared__ uint32_t cnt[kSortBins];
    cnt[threadIdx.x] = 0;
    __syncthreads();
    const uint32_t base = blockIdx.x * kSortTile;
    #pragma unroll
    for (int k = 0; k < kSortItems; ++k) {
        const uint32_t i = base + k * kSortThreads + threadIdx.x;
        if (i < n) atomicAdd(&cnt[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[size_t(threadIdx.x) * tiles + blockIdx.x] = cnt[threadIdx.x];
}

// Exclusive prefix sum of in[0, m) into out (in == out allowed), m up to
// kScanChunk * kScanThreads: scan_reduce_kernel sums each kScanChunk-element
// chunk, scan_top_kernel scans the chunk sums in one block, and
// scan_down_kernel scans each chunk (four consecutive elements per thread,
// a shuffle scan per warp, then across warps) and adds its chunk's prefix.
constexpr int kScanThreads = 1024;
constexpr int kScanChunk = 4 * kScanThreads;

// Inclusive scan of v across the block (1024 threads); every thread gets
// its own inclusive prefix.
__device__ __forceinline__ uint32_t block_scan_inclusive(uint32_t v, uint32_t* warp_sums) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    #pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const uint32_t u = __shfl_up_sync(0xffffffffu, v, off);
        if (lane >= off) v += u;
    }
    if (lane == 31) warp_sums[w] = v;
    __syncthreads();
    if (w == 0) {
        uint32_t s = warp_sums[lane];
        #pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const uint32_t u = __shfl_up_sync(0xffffffffu, s, off);
            if (lane >= off) s += u;
        }
        warp_sums[lane] = s;
    }
    __syncthreads();
    return v + (w > 0 ? warp_sums[w - 1] : 0u);
}

__global__ void __launch_bounds__(kScanThreads) scan_reduce_kernel(const uint32_t* __restrict__ in, uint32_t m,
                                                                   uint32_t* __restrict__ sums) {
    __shared__ uint32_t red[kScanThreads / 32];
    const uint32_t base = blockIdx.x * kScanChunk;
    uint32_t s = 0;
    #pragma unroll
    for (int k = 0; k < 4; ++k) {
        const uint32_t i = base + k * kScanThreads + threadIdx.x;
        if (i < m) s += in[i];
    }
    #pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x < 32) {
        uint32_t v = red[threadIdx.x];
        #pragma unroll
        for (int off = 16; off > 0; off >>= 1) v += __shfl_xor_sync(0xffffffffu, v, off);
        if (threadIdx.x == 0) sums[blockIdx.x] = v;
    }
}

__global__ void __launch_bounds__(kScanThreads) scan_top_kernel(uint32_t* sums, uint32_t chunks) {
    __shared__ uint32_t ws[kScanThreads / 32];
    const uint32_t v = threadIdx.x < chunks ? sums[threadIdx.x] : 0u;
    const uint32_t inc = block_scan_inclusive(v, ws);
    if (threadIdx.x < chunks) sums[threadIdx.x] = inc - v;
}

__global__ void __launch_bounds__(kScanThreads) scan_down_kernel(const uint32_t* in, uint32_t* out, uint32_t m,
                                                                 const uint32_t* __restrict__ sums) {
    __shared__ uint32_t ws[kScanThreads / 32];
    const uint32_t i0 = blockIdx.x * kScanChunk + threadIdx.x * 4;
    uint32_t x[4];
    #pragma unroll
    for (int k = 0; k < 4; ++k) x[k] = i0 + k < m ? in[i0 + k] : 0u;
    const uint32_t local = x[0] + x[1] + x[2] + x[3];
    const uint32_t inc = block_scan_inclusive(local, ws);
    uint32_t run = sums[blockIdx.x] + inc - local;
    #pragma unroll
    for (int k = 0; k < 4; ++k) {
        if (i0 + k < m) out[i0 + k] = run;
        run += x[k];
    }
}

// Host side: the three launches of an exclusive scan of m elements (m up to
// kScanChunk * kScanThreads); sums holds m / kScanChunk + 1 words.
inline void scan_exclusive(const uint32_t* in, uint32_t* out, uint32_t m, uint32_t* sums, cudaStream_t stream) {
    if (m == 0) return;
    const uint32_t chunks = (m + kScanChunk - 1) / kScanChunk;
    scan_reduce_kernel<<<chunks, kScanThreads, 0, stream>>>(in, m, sums);
    scan_top_kernel<<<1, kScanThreads, 0, stream>>>(sums, chunks);
    scan_down_kernel<<<chunks, kScanThreads, 0, stream>>>(in, out, m, sums);
}

__global__ void __launch_bounds__(kSortThreads) sort_scatter_kernel(const uint32_t* __restrict__ keys_in,
                                                                    const uint32_t* __restrict__ vals_in,
                                                                    uint32_t* __restrict__ keys_out,
                                                                    uint32_t* __restrict__ vals_out, uint32_t n,
                                                                    int shift, uint32_t tiles,
                                                                    const uint32_t* __restrict__ offs) {
    __shared__ uint32_t whist[kSortWarps][kSortBins];   // per-warp digit counts, then per-warp bases
    __shared__ uint32_t tile_off[kSortBins];
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    for (int q = t; q < kSortWarps * kSortBins; q += kSortThreads) (&whist[0][0])[q] = 0u;
    tile_off[t] = offs[size_t(t) * tiles + blockIdx.x];
    const uint32_t wbase = blockIdx.x * kSortTile + uint32_t(w) * 32u * kSortItems;
    uint32_t key[kSortItems], val[kSortItems];
    #pragma unroll
    for (int c = 0; c < kSortItems; ++c) {
        const uint32_t i = wbase + c * 32 + lane;
        key[c] = i < n ? keys_in[i] : 0u;
        val[c] = i < n ? vals_in[i] : 0u;
    }
    __syncthreads();
    const uint32_t lt = (1u << lane) - 1u;
    // sweep 1: the warp's digit counts (one lane per group of equal digits adds)
    #pragma unroll
    for (int c = 0; c < kSortItems; ++c) {
        const bool valid = wbase + c * 32 + lane < n;
        const uint32_t mask = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const uint32_t d = (key[c] >> shift) & 255u;
            const uint32_t peers = __match_any_sync(mask, d);
            if ((peers & lt) == 0u) whist[w][d] += __popc(peers);
        }
        __syncwarp();
    }
    __syncthreads();
    {   // per digit, the counts of the earlier warps
        uint32_t run = 0;
        #pragma unroll
        for (int v = 0; v < kSortWarps; ++v) {
            const uint32_t c = whist[v][t];
            whist[v][t] = run;
            run += c;
        }
    }
    __syncthreads();
    // sweep 2: positions in chunk order, lane order within a chunk
    #pragma unroll
    for (int c = 0; c < kSortItems; ++c) {
        const bool valid = wbase + c * 32 + lane < n;
        const uint32_t mask = __ballot_sync(0xffffffffu, valid);
        uint32_t d = 0, peers = 0;
        if (valid) {
            d = (key[c] >> shift) & 255u;
            peers = __match_any_sync(mask, d);
            const uint32_t pos = tile_off[d] + whist[w][d] + __popc(peers & lt);
            keys_out[pos] = key[c];
            vals_out[pos] = val[c];
        }
        __syncwarp();
        if (valid && (peers & lt) == 0u) whist[w][d] += __popc(peers);
        __syncwarp();
    }
}

} // namespace rr

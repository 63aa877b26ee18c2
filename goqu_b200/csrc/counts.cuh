// Shot histograms on the device: the sampled indices of one call become
// (outcome, count) pairs in increasing outcome order, the content of the
// map[bitstring]int that goqu's Run returns (sim/statevector/sim.go:40-58,
// formatBitstring :306-316), so a caller builds its map in O(distinct
// outcomes) instead of O(shots).
//
// Method: a stable least-significant-digit radix sort of the indices with
// 8-bit digits over only the index's significant bits (ceil(n / 8) passes for
// 2^n outcomes), then a run-length encoding. Each sort pass is three
// launches: per-tile digit counts (digit-major, so one exclusive scan gives
// every tile's output offset per digit), the scan, and a scatter that ranks
// each key among the equal digits before it in its tile (warp match plus a
// per-digit prefix over warps), which keeps the pass stable. Deterministic:
// no step depends on the order in which threads run.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

namespace gq {

constexpr int kHistThreads = 256;
constexpr int kHistRounds = 4;                               // keys per thread per tile
constexpr int kHistTile = kHistThreads * kHistRounds;        // keys per tile
constexpr int kHistWarps = kHistThreads / 32;

__device__ __forceinline__ uint32_t hist_digit(uint64_t k, int shift) { return (uint32_t)(k >> shift) & 255u; }

// counts[d * ntiles + tile] = keys of the tile whose digit is d.
__global__ void __launch_bounds__(kHistThreads) k_radix_counts(const uint64_t* __restrict__ keys, uint64_t n,
                                                               int shift, uint32_t ntiles,
                                                               uint32_t* __restrict__ counts) {
    __shared__ uint32_t h[256];
    h[threadIdx.x] = 0;
    __syncthreads();
    const uint64_t base = (uint64_t)blockIdx.x * kHistTile;
    for (int r = 0; r < kHistRounds; ++r) {
        const uint64_t i = base + (uint64_t)r * kHistThreads + threadIdx.x;
        if (i < n) atomicAdd(&h[hist_digit(keys[i], shift)], 1u);
    }
    __syncthreads();
    counts[(uint64_t)threadIdx.x * ntiles + blockIdx.x] = h[threadIdx.x];
}

// Exclusive prefix sum of x[0, len) in place (one block of 1024 threads, each
// scanning a contiguous segment); *total receives the sum when non-null.
__global__ void __launch_bounds__(1024) k_scan_u32(uint32_t* __restrict__ x, uint64_t len, uint32_t* total) {
    __shared__ uint32_t part[1024];
    const uint64_t per = (len + 1023) / 1024;
    const uint64_t lo = min(len, per * threadIdx.x), hi = min(len, lo + per);
    uint32_t s = 0;
    for (uint64_t i = lo; i < hi; ++i) s += x[i];
    part[threadIdx.x] = s;
    __syncthreads();
    for (int o = 1; o < 1024; o <<= 1) {  // inclusive Hillis-Steele scan of the segment sums
        const uint32_t v = threadIdx.x >= (unsigned)o ? part[threadIdx.x - o] : 0u;
        __syncthreads();
        part[threadIdx.x] += v;
        __syncthreads();
    }
    uint32_t run = threadIdx.x ? part[threadIdx.x - 1] : 0u;
    for (uint64_t i = lo; i < hi; ++i) {
        const uint32_t v = x[i];
        x[i] = run;
        run += v;
    }
    if (total && threadIdx.x == 1023) *total = part[1023];
}

// Stable scatter of one radix pass: out[offset(digit, tile) + rank] = key,
// rank = keys of the same digit earlier in the tile.
__global__ void __launch_bounds__(kHistThreads) k_radix_scatter(const uint64_t* __restrict__ keys, uint64_t n,
                                                                int shift, uint32_t ntiles,
                                                                const uint32_t* __restrict__ offsets,
                                                                uint64_t* __restrict__ out) {
    __shared__ uint32_t off[256];
    __shared__ uint32_t wcnt[kHistWarps][256];
    const int t = threadIdx.x, w = t >> 5, lane = t & 31;
    off[t] = offsets[(uint64_t)t * ntiles + blockIdx.x];
    const uint64_t base = (uint64_t)blockIdx.x * kHistTile;
    const uint32_t lt_mask = (1u << lane) - 1u;
    for (int r = 0; r < kHistRounds; ++r) {
        for (int k = 0; k < kHistWarps; ++k) wcnt[k][t] = 0;
        const uint64_t i = base + (uint64_t)r * kHistThreads + t;
        const bool valid = i < n;
        const uint64_t key = valid ? keys[i] : 0;
        const uint32_t d = valid ? hist_digit(key, shift) : 256u;  // 256: no key
        __syncthreads();
        const uint32_t same = __match_any_sync(0xffffffffu, d);
        const uint32_t before = __popc(same & lt_mask);
        if (valid && before == 0) wcnt[w][d] = __popc(same);
        __syncthreads();
        // per digit: exclusive prefix over the warps, continuing the tile's count
        uint32_t acc = off[t];
        for (int k = 0; k < kHistWarps; ++k) {
            const uint32_t c = wcnt[k][t];
            wcnt[k][t] = acc;
            acc += c;
        }
        off[t] = acc;
        __syncthreads();
        if (valid) out[wcnt[w][d] + before] = key;
        __syncthreads();
    }
}

// Run starts of sorted keys: flag[i] = 1 where key[i] differs from key[i-1].
__global__ void k_run_flags(const uint64_t* __restrict__ keys, uint64_t n, uint32_t* __restrict__ flag) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        flag[i] = (i == 0 || keys[i] != keys[i - 1]) ? 1u : 0u;
}

// After the exclusive scan of the flags (pos), run j starts at the index i
// with flag and pos[i] = j: outcome[j] = key[i], start[j] = i.
__global__ void k_run_starts(const uint64_t* __restrict__ keys, uint64_t n, const uint32_t* __restrict__ pos,
                             uint64_t* __restrict__ outcome, uint64_t* __restrict__ start) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const bool first = i == 0 || keys[i] != keys[i - 1];
        if (first) {
            outcome[pos[i]] = keys[i];
            start[pos[i]] = i;
        }
    }
}

// count[j] = start[j + 1] - start[j], the last run ending at n; *nruns is
// the number of runs (the scan's total).
__global__ void k_run_counts(const uint64_t* __restrict__ start, uint64_t n, const uint32_t* __restrict__ nruns,
                             uint64_t* __restrict__ count) {
    const uint64_t d = *nruns;
    for (uint64_t j = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; j < d; j += (uint64_t)gridDim.x * blockDim.x)
        count[j] = (j + 1 < d ? start[j + 1] : n) - start[j];
}

}  // namespace gq

// dsmc_radix.cuh -- stable LSD radix sort of cell ids (8-bit digits) for the full sorts.
//
// The full sorts (dsmc_init_cloud / dsmc_set_state, and dsmc_sort_cells_noalloc) order atoms
// stably by (cell, input index).  Each pass over one digit counts the digit per chunk of
// RADIX_CHUNK keys (radix_hist), takes an exclusive scan of the digit-major count table (the
// caller's scan: digit d of chunk b lands after every smaller digit and after digit d of every
// earlier chunk), then writes each key to its place (radix_scatter), ranking equal digits in
// input order inside the chunk.  Every pass is stable, so after the passes over all digits of
// the largest cell id the order is by cell and, within a cell, by input index.  The cost is
// O(n) per pass whatever the cells hold: one cell holding every atom sorts as fast as any
// other distribution.
#ifndef DSMC_RADIX_CUH
#define DSMC_RADIX_CUH

#include <cuda_runtime.h>
#include <stdint.h>

namespace dsmc {

constexpr int RADIX_BITS = 8;
constexpr int RADIX_DIGITS = 1 << RADIX_BITS;
constexpr int RADIX_BLOCK = 256;                // threads of the radix kernels
constexpr int RADIX_ROUNDS = 16;                // rounds of RADIX_BLOCK keys per chunk
constexpr int RADIX_CHUNK = RADIX_BLOCK * RADIX_ROUNDS;
static_assert(RADIX_BLOCK == RADIX_DIGITS, "one thread per digit in the per-round bookkeeping");

// chunks of n keys, and the size of the digit-major count table
inline int radix_chunks(int n) { return (n + RADIX_CHUNK - 1) / RADIX_CHUNK; }
inline int64_t radix_table(int n) { return (int64_t)RADIX_DIGITS * (int64_t)(radix_chunks(n) > 0 ? radix_chunks(n) : 1); }
// passes over 8-bit digits that cover every id below `ids` (at least one)
inline int radix_passes(int ids) {
    int bits = 0;
    while (bits < 31 && (1ll << bits) < (long long)ids) ++bits;
    const int p = (bits + RADIX_BITS - 1) / RADIX_BITS;
    return p > 0 ? p : 1;
}

// table[d * nchunks + b] = keys of chunk b whose digit at `shift` is d.  (The kernels are static:
// each translation unit that includes this header has its own copy.)
static __global__ void __launch_bounds__(RADIX_BLOCK) radix_hist(const int* __restrict__ key, int n, int shift,
                                                          int* __restrict__ table, int nchunks) {
    __shared__ int h[RADIX_DIGITS];
    h[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * RADIX_CHUNK;
#pragma unroll 4
    for (int r = 0; r < RADIX_ROUNDS; ++r) {
        const int j = base + r * RADIX_BLOCK + threadIdx.x;
        if (j < n) atomicAdd(&h[((unsigned)key[j] >> shift) & (RADIX_DIGITS - 1)], 1);
    }
    __syncthreads();
    table[(size_t)threadIdx.x * nchunks + blockIdx.x] = h[threadIdx.x];
}

// Writes chunk b's keys (and values; the input index when val_in is null) to key_out/val_out at
// off[d * nchunks + b] + (earlier keys of the chunk with digit d).  Keys go round by round
// (RADIX_BLOCK consecutive keys); in a round a key's rank among equal digits is the count in
// earlier warps plus the count in earlier lanes of its own warp.  key_out may be null (the last
// pass needs only the values).
static __global__ void __launch_bounds__(RADIX_BLOCK) radix_scatter(const int* __restrict__ key_in,
                                                             const int* __restrict__ val_in, int n, int shift,
                                                             const int* __restrict__ off, int nchunks,
                                                             int* __restrict__ key_out, int* __restrict__ val_out) {
    constexpr int NW = RADIX_BLOCK / 32;
    __shared__ int base[RADIX_DIGITS];
    __shared__ int wcnt[NW][RADIX_DIGITS];
    const int t = threadIdx.x, lane = t & 31, warp = t >> 5;
    base[t] = off[(size_t)t * nchunks + blockIdx.x];
    const int b0 = blockIdx.x * RADIX_CHUNK;
    for (int r = 0; r < RADIX_ROUNDS; ++r) {
        const int j = b0 + r * RADIX_BLOCK + t;
        const bool valid = j < n;
        const int k = valid ? key_in[j] : 0;
        const int v = valid ? (val_in ? val_in[j] : j) : 0;
        const int d = valid ? (int)(((unsigned)k >> shift) & (RADIX_DIGITS - 1)) : RADIX_DIGITS;  // padding apart
#pragma unroll
        for (int w = 0; w < NW; ++w) wcnt[w][t] = 0;
        __syncthreads();  // cleared counts (and, in round 0, base) visible
        const unsigned peers = __match_any_sync(0xffffffffu, d);
        const int lrank = __popc(peers & ((1u << lane) - 1u));
        if (valid && lrank == 0) wcnt[warp][d] = __popc(peers);
        __syncthreads();
        if (valid) {
            int pre = 0;
            for (int w = 0; w < warp; ++w) pre += wcnt[w][d];
            const int dest = base[d] + pre + lrank;
            if (key_out) key_out[dest] = k;
            val_out[dest] = v;
        }
        __syncthreads();  // every thread has read base before it advances
        int tot = 0;
#pragma unroll
        for (int w = 0; w < NW; ++w) tot += wcnt[w][t];
        base[t] += tot;
        // the next round's clear follows the barrier below it, after these reads
        __syncthreads();
    }
}

}  // namespace dsmc

#endif  // DSMC_RADIX_CUH

// dsmc_kernels.cuh -- sm_100a kernels of one DSMC timestep.
//
// Data layout in HBM (per precision R = float | double, R4 = float4 | double4):
//   pos[i] = (x, y, z, atom id bits)   vel[i] = (vx, vy, vz, flag bits)   psi[i] = (u_re, u_im, d_re, d_im)
//   three structure-of-arrays streams of 16 B (FP32) per atom, double-buffered, plus a
//   permutation src[] (4 B per atom): the atom in sorted position j is stored at src[j].  The
//   sorted order groups atoms by global cell (clouds one after another, each cloud's grid cells
//   then its overflow cell), so every cell is a contiguous range [start[c], start[c+1]) of j.
//
// One step = 4 launches with static grids, captured in a CUDA graph of two steps:
//   step_pass        per tile of ~T sorted positions: gather the atoms through src, collide the
//                    tile's cells in shared memory, then move + spin + evaporate every atom once,
//                    write the new state at its current position j (coalesced) with an 8-byte
//                    sort key (stayers ranked in their cell by warp ballots), count leavers L[c] /
//                    incoming movers I[c] (fire-and-forget atomics), list movers in per-warp
//                    chunks of the step's mover list, and add exact totals into per-cloud
//                    buckets.  The only heavy pass: the step is computed once.
//   scan_cells       one-pass scan (decoupled look-back) of the per-cell counts n_c - L_c + I_c:
//                    new start[], movers' base slots, largest cell, the next tiling of a single
//                    cloud; its last block runs the top level (next tile size, per-cloud starts
//                    and tile offsets); extra blocks compute the overflow-cell carries and close
//                    each cloud's step totals (diagnostics, knife temperature, step counter)
//   permute_pass     the next permutation src'[dest] = j for the stayers (4 B per atom instead of
//                    moving 48 B), each incoming mover's slot in its cell's incoming list, and
//                    (batched clouds, or a changed tile size) the next tiling's starts from the
//                    atoms placed at cell starts
//   mover_rank       deterministic rank of each incoming mover by its old position -> src'
// The new order is the stable sort by (new cell, moved?, old position): in each new cell the atoms
// that stayed keep their order, followed by the atoms that entered it, by old position.  Tiles are
// contiguous, cloud-pure ranges of sorted positions whose boundaries snap to cell starts (the
// overflow cell, which never collides, is split at nominal boundaries).
#ifndef DSMC_KERNELS_CUH
#define DSMC_KERNELS_CUH

#include <cuda_runtime.h>
#include "dsmc_physics.h"
#include "dsmc_radix.cuh"

namespace dsmc {

template <class R> struct V4T;
template <> struct V4T<float> { typedef float4 type; };
template <> struct V4T<double> { typedef double4 type; };

enum : int {
    EB_CELL_FULL = 1,
    EB_NAN = 2,
    EB_CAPACITY = 4,
    EB_INIT_REJECT = 8,
    EB_TILE_OVERFLOW = 16,
    EB_INCONSISTENT = 32,
    EB_TIMEOUT = 64,
    EB_LOG_FULL = 128
};

constexpr int MOVER_GRID = 148 * 8;
// step_pass hands out mover-list slots from per-warp chunks of MV_CHUNK, each reserved with one
// atomic on the step's mover counter (one contended atomic per 64 movers instead of one per warp
// pass with a mover); a warp's last chunk leaves up to MV_CHUNK - 1 unused slots, marked as holes
// (cell -1), so the list holds up to capacity + MV_CHUNK x (resident step_pass warps) entries
constexpr int MV_CHUNK = 64;  // grid-stride kernels over the mover list

struct __align__(16) TilePartial {
    i128 sum_v2, sum_B, evap_v2, evap_B;
    long long n_alive, n_maj, n_knife, coll, cand, pad0, pad1, pad2;
};

// Per-cloud totals of one step, gathered in ACC_BUCKETS buckets per cloud (tile b adds into bucket
// b mod ACC_BUCKETS) with 64-bit atomic adds whose results are not read.  Each 128-bit sum (all of
// them non-negative, below 2^126) is split into three 42-bit limbs, so a bucket's limb sum cannot
// wrap before 2^21 tiles.  finalize recombines and clears the buckets.
constexpr int ACC_BUCKETS = 16;

// smallest nominal tile (sizes the tile tables: at most capacity / MIN_TILE + clouds + 2 tiles)
constexpr int MIN_TILE = 128;
// A grid cell of more than dense_threshold(CAP) atoms is dense: like the overflow cell it is split
// across tiles (a tile begins at each nominal start inside it), and dense_collide collides it
// before step_pass, reaching its atoms through the sorted order.  A tiling of nominal size T holds
// tiles of at most T - 1 + (largest other grid cell) atoms, so the scan's T = CAP + 1 - that
// count never falls below DENSE_MIN_TILE (cells fuller than that go to dense_collide, which
// stages a cell in shared memory, rather than shrinking every tile of the step).
constexpr int DENSE_MIN_TILE = 512;
__host__ __device__ constexpr int dense_threshold(int cap) { return cap + 1 - DENSE_MIN_TILE; }
// tile_ovf word of a tile: the stayers of its last cell when that cell continues into the next
// tile, and TILE_WHOLE when the tile lies inside that cell (it also began inside it)
constexpr int TILE_WHOLE = 1 << 30;
struct __align__(16) CloudAccum {
    unsigned long long v2[3], B[3], ev2[3], eB[3];
    unsigned long long n_alive, n_maj, n_knife, coll, cand, pad[3];
};

struct CloudDyn {
    int n[2];         // atoms, by parity
    int start[2];     // first atom index, by parity
    int tile_off[2];  // first tile, by parity
    int ntiles[2];
    double T_knife;   // temperature used by the knife of the coming step
    double pad;
};

struct __align__(16) CloudDiagDev {
    i128 sum_v2, sum_B, cum_evap_v2, cum_evap_B;
    long long step, n_alive, cum_evap, cum_maj, cum_knife, cum_coll, cum_cand, err, cum_atom_steps, pad;
};

struct Ctl {
    int n[2];
    int ntiles[2];
    int step[2];
    int err;
    int movers[2];  // movers listed by the step of each parity (the other parity's is cleared by the scan)
    int novf[2];    // tiles listed in ovf_list by the step of each parity
    int scan_done;    // scan_cells blocks finished (the last one runs the top level and clears it)
    int max_cell;     // largest coming grid-cell count, gathered by scan_cells (cleared by its top level)
    int tile_T[2];    // nominal tile size of the tiling built for each parity
    int scan_ticket;  // scan_cells blocks started: a block's ticket is the scan block it processes
    int tiles_built[2];  // 1: scan_cells wrote the tiling of that parity (else the atoms' placement does)
    unsigned scan_epoch;  // scan_cells launches completed: tags the look-back descriptors of a launch
    int ndense[2];  // dense grid cells listed for the step of each parity (collided by dense_collide;
                    // listed where the atoms are placed, the list of the coming step cleared by the scan)
};

// keys written by step_pass, one per atom position:
//   .y = kind | KEY_OVF_CELL | (rank << KEY_RANK_SHIFT) | (cloud << KEY_CLOUD_SHIFT)
//   KIND_STAY  .x = cell, rank among the cell's stayers before it (the cell starts in this tile)
//   KIND_OVF   .x = tile, rank among the tile's stayers of the split cell (overflow or dense)
//              that the tile begins inside (tile_cell), which started in an earlier tile
//   KIND_MOVE  .x = slot in the step's mover list;  KIND_LOST  .x = -1
//   KEY_OVF_CELL: the stayer's cell is its cloud's overflow cell
// A stayer's rank counts positions of its tile, so it is below the staging capacity (< 2^11); the
// cloud rides along so that permute_pass need not search for the cell's cloud.
enum : int { KIND_STAY = 0, KIND_MOVE = 1, KIND_LOST = 2, KIND_OVF = 3 };
constexpr int KEY_OVF_CELL = 4;
constexpr int KEY_RANK_SHIFT = 3;
constexpr int KEY_RANK_BITS = 11;
constexpr int KEY_RANK_MASK = (1 << KEY_RANK_BITS) - 1;
constexpr int KEY_CLOUD_SHIFT = KEY_RANK_SHIFT + KEY_RANK_BITS;
constexpr int KEY_MAX_CLOUDS = 1 << (31 - KEY_CLOUD_SHIFT);  // clouds a handle may hold
// mover records written by step_pass: .x = target cell (-1: an unused slot of a warp's chunk),
// .y = old position, .z unused, .w = cloud | MREC_OVF_CELL when the target is the cloud's overflow cell
constexpr int MREC_OVF_CELL = 1 << 30;

__device__ __forceinline__ int2 stayer_key(bool split_ovf, int tile, int cell, int rank, bool ovf_cell, int cloud) {
    const int tail = (rank << KEY_RANK_SHIFT) | (cloud << KEY_CLOUD_SHIFT);
    return make_int2(split_ovf ? tile : cell, (split_ovf ? KIND_OVF : KIND_STAY) | (ovf_cell ? KEY_OVF_CELL : 0) | tail);
}

template <class R> struct Args {
    typedef typename V4T<R>::type R4;
    const R4* pos_in;
    const R4* vel_in;
    const R4* psi_in;
    R4* pos_out;
    R4* vel_out;
    R4* psi_out;
    const int* src_in;   // sorted position -> storage index of the current state
    int* src_out;        // the same for the state this step writes
    int2* keys;          // per current position: sort key written by step_pass
    const int* old_start;
    int* new_start;
    int* Lc;
    int* Ic;
    int* mover_base;
    R* sigvrmax;
    int4* mrec;
    int mrec_cap;  // entries of the mover list (atoms of capacity + the warps' chunk slack)
    int* in_list;
    const int* tile_begin;
    const int* tile_cloud;
    const int* tile_split;  // 1: the tile begins inside a cell (overflow or dense) that began earlier
    int* tile_begin_next;
    int* tile_cloud_next;
    int* tile_split_next;
    int* tile_ovf;
    int* tile_ovf_carry;
    int* ovf_list;  // split tiles and tiles whose last cell continues, in any order (ctl->novf[parity])
    int* tile_cell;  // per split tile: the cell it begins inside (written by step_pass)
    int2* dense_list;  // (cell, cloud) of each dense grid cell of the coming step (ctl->ndense)
    int dense_cap;
    // per cloud: atoms the step removed (Majorana, knife, or an unstageable tile), counted per tile
    // by step_pass; the cell scan starts each cloud's look-back chain from the earlier clouds' old
    // totals less these (atoms never change clouds), and its top level clears them
    int* cloud_lost;
    CloudAccum* accum;  // nclouds x ACC_BUCKETS
    const CloudPhys<R>* clouds;
    CloudPhys<R> one;   // the parameters of cloud 0, read from the kernel parameters by one-cloud runs
    CloudDyn* cdyn;
    CloudDiagDev* cdiag;
    Ctl* ctl;
    unsigned long long* scan_desc;  // look-back descriptor of each scan block (LB_STRIDE apart)
    const int* cloud_cell_base;     // first cell of each cloud, nclouds + 1
    const int4* scan_blk;  // per scan block: cloud, first cell, end of the cloud's cells, end of the block's
    const int* cloud_first_blk;  // nclouds + 1
    int nclouds, total_cells, nscan_blocks, max_tiles, tile_nominal, collide_every, parity, init_mode;
    int tile_cap;  // atoms a tile can stage (CAP): a tiling of nominal size T fits cells of CAP - T + 1
    int tile_pass;  // atoms one step_pass block handles per pass (its thread count)
    int tile_fill;  // > 0 (the resident step_pass blocks): shrink the nominal size for small runs
    int capacity;
    // collision record (adjoint runs): pairs by atom id, directions, per-step offsets
    int2* clog_ij;
    double* clog_n;
    int* clog_count;
    int* clog_off;
    int clog_cap, clog_step0, clog_steps;
    // snapshot records (null when off): per atom id slot (cloud's id_base + id) the state at the
    // step it was lost -- position with the step number in the fourth lane, velocity with the fate
    // -- and per global cell (step, accepted collisions) of the last step that collided it
    R4* rec_evap_pos;
    R4* rec_evap_vel;
    int2* rec_cell_coll;
    unsigned long long seed;
};

// ---------------------------------------------------------------------------------------------
// block-wide helpers
// ---------------------------------------------------------------------------------------------
template <int BLOCK>
__device__ __forceinline__ uint32_t block_excl_scan_u32(uint32_t v, uint32_t* wsum, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = BLOCK / 32;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < NW ? wsum[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < NW) wsum[lane] = w;
    }
    __syncthreads();
    uint32_t off = warp ? wsum[warp - 1] : 0u;
    total = wsum[NW - 1];
    __syncthreads();
    return off + x - v;
}

__device__ __forceinline__ i128 shfl_down_i128(i128 v, int o) {
    unsigned long long lo = (unsigned long long)v;
    long long hi = (long long)(v >> 64);
    lo = __shfl_down_sync(0xffffffffu, lo, o);
    hi = __shfl_down_sync(0xffffffffu, hi, o);
    return (i128)(((unsigned __int128)(unsigned long long)hi << 64) | (unsigned __int128)lo);
}
__device__ __forceinline__ i128 warp_sum_i128(i128 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += shfl_down_i128(v, o);
    return v;
}
__device__ __forceinline__ long long warp_sum_ll(long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    return v;
}

// Exact warp sum of non-negative 128-bit values: five 26-bit limbs (the top one 24 bits), each
// summed over the 32 lanes by redux.sync without overflow (32 x 2^26 < 2^32), recombined mod 2^128.
__device__ __forceinline__ i128 warp_sum_u128_redux(i128 v) {
    const unsigned long long lo = (unsigned long long)v;
    const unsigned long long hi = (unsigned long long)((unsigned __int128)v >> 64);
    constexpr unsigned M26 = (1u << 26) - 1u;
    const unsigned s0 = __reduce_add_sync(0xffffffffu, (unsigned)lo & M26);
    const unsigned s1 = __reduce_add_sync(0xffffffffu, (unsigned)(lo >> 26) & M26);
    const unsigned s2 = __reduce_add_sync(0xffffffffu, (unsigned)((lo >> 52) | (hi << 12)) & M26);
    const unsigned s3 = __reduce_add_sync(0xffffffffu, (unsigned)(hi >> 14) & M26);
    const unsigned s4 = __reduce_add_sync(0xffffffffu, (unsigned)(hi >> 40));
    const unsigned __int128 r = (unsigned __int128)s0 + ((unsigned __int128)s1 << 26) +
                                ((unsigned __int128)s2 << 52) + ((unsigned __int128)s3 << 78) +
                                ((unsigned __int128)s4 << 104);
    return (i128)r;
}

// per-thread accumulators of step_pass (the retained atoms and the collisions) and their block
// reduction; lost atoms are rare and go straight into a block-shared LostAcc
struct StepAcc {
    i128 sum_v2, sum_B;
    unsigned n_alive, coll, cand;
};
struct LostAcc {
    unsigned long long ev2[3], eB[3], n_maj, n_knife;
};
__device__ __forceinline__ void zero_acc(StepAcc& a) {
    a.sum_v2 = 0; a.sum_B = 0;
    a.n_alive = 0; a.coll = 0; a.cand = 0;
}
__device__ __forceinline__ void warp_reduce_acc(StepAcc& a) {
    a.sum_v2 = warp_sum_u128_redux(a.sum_v2);
    a.sum_B = warp_sum_u128_redux(a.sum_B);
    a.n_alive = __reduce_add_sync(0xffffffffu, a.n_alive);
    a.coll = __reduce_add_sync(0xffffffffu, a.coll);
    a.cand = __reduce_add_sync(0xffffffffu, a.cand);
}
// every thread of the block calls; thread 0 receives the block total in `out`
template <int BLOCK>
__device__ __forceinline__ void block_reduce_acc(StepAcc& a, StepAcc* sm, TilePartial& out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = BLOCK / 32;
    static_assert(NW <= 32, "one warp reduces the warp totals");
    warp_reduce_acc(a);
    if (lane == 0) sm[warp] = a;
    __syncthreads();
    if (warp == 0) {
        StepAcc w;
        if (lane < NW) w = sm[lane]; else zero_acc(w);
        warp_reduce_acc(w);
        if (lane == 0) {
            out.sum_v2 = w.sum_v2; out.sum_B = w.sum_B; out.evap_v2 = 0; out.evap_B = 0;
            out.n_alive = w.n_alive; out.n_maj = 0; out.n_knife = 0;
            out.coll = w.coll; out.cand = w.cand; out.pad0 = 0;
            out.pad1 = 0; out.pad2 = 0;
        }
    }
}

// reduce 4 i128 + 5 int64 over the block into p (thread 0 holds the result)
template <int BLOCK>
__device__ __forceinline__ void block_reduce_partial(TilePartial& t, TilePartial* sm) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = BLOCK / 32;
    t.sum_v2 = warp_sum_i128(t.sum_v2);
    t.sum_B = warp_sum_i128(t.sum_B);
    t.evap_v2 = warp_sum_i128(t.evap_v2);
    t.evap_B = warp_sum_i128(t.evap_B);
    t.n_alive = warp_sum_ll(t.n_alive);
    t.n_maj = warp_sum_ll(t.n_maj);
    t.n_knife = warp_sum_ll(t.n_knife);
    t.coll = warp_sum_ll(t.coll);
    t.cand = warp_sum_ll(t.cand);
    if (lane == 0) sm[warp] = t;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int w = 1; w < NW; ++w) {
            t.sum_v2 += sm[w].sum_v2;
            t.sum_B += sm[w].sum_B;
            t.evap_v2 += sm[w].evap_v2;
            t.evap_B += sm[w].evap_B;
            t.n_alive += sm[w].n_alive;
            t.n_maj += sm[w].n_maj;
            t.n_knife += sm[w].n_knife;
            t.coll += sm[w].coll;
            t.cand += sm[w].cand;
        }
    }
    __syncthreads();
}

__device__ __forceinline__ void add_limbs(unsigned long long* dst, i128 v) {
    const unsigned __int128 u = (unsigned __int128)v;
    constexpr unsigned long long M42 = (1ull << 42) - 1ull;
    if (u == 0) return;
    atomicAdd(dst, (unsigned long long)u & M42);
    atomicAdd(dst + 1, (unsigned long long)(u >> 42) & M42);
    atomicAdd(dst + 2, (unsigned long long)(u >> 84));
}
// one tile's totals into its cloud's bucket (one thread)
__device__ __forceinline__ void accum_tile(CloudAccum* bucket, const TilePartial& t) {
    add_limbs(bucket->v2, t.sum_v2);
    add_limbs(bucket->B, t.sum_B);
    add_limbs(bucket->ev2, t.evap_v2);
    add_limbs(bucket->eB, t.evap_B);
    if (t.n_alive) atomicAdd(&bucket->n_alive, (unsigned long long)t.n_alive);
    if (t.n_maj) atomicAdd(&bucket->n_maj, (unsigned long long)t.n_maj);
    if (t.n_knife) atomicAdd(&bucket->n_knife, (unsigned long long)t.n_knife);
    if (t.coll) atomicAdd(&bucket->coll, (unsigned long long)t.coll);
    if (t.cand) atomicAdd(&bucket->cand, (unsigned long long)t.cand);
}
// a block's lost-atom totals into a bucket (one thread), then cleared
__device__ __forceinline__ void accum_lost(CloudAccum* bucket, LostAcc& s) {
    for (int i = 0; i < 3; ++i) {
        if (s.ev2[i]) atomicAdd(&bucket->ev2[i], s.ev2[i]);
        if (s.eB[i]) atomicAdd(&bucket->eB[i], s.eB[i]);
        s.ev2[i] = 0;
        s.eB[i] = 0;
    }
    if (s.n_maj) atomicAdd(&bucket->n_maj, s.n_maj);
    if (s.n_knife) atomicAdd(&bucket->n_knife, s.n_knife);
    s.n_maj = 0;
    s.n_knife = 0;
}
__device__ __forceinline__ i128 from_limbs(const unsigned long long* l) {
    return (i128)((unsigned __int128)l[0] + ((unsigned __int128)l[1] << 42) + ((unsigned __int128)l[2] << 84));
}

__device__ __forceinline__ void zero_partial(TilePartial& t) {
    t.sum_v2 = 0; t.sum_B = 0; t.evap_v2 = 0; t.evap_B = 0;
    t.n_alive = 0; t.n_maj = 0; t.n_knife = 0; t.coll = 0; t.cand = 0;
    t.pad0 = 0; t.pad1 = 0; t.pad2 = 0;
}

template <class R>
__device__ __forceinline__ void load_cloud(CloudPhys<R>& dst, const CloudPhys<R>* src) {
    static_assert(sizeof(CloudPhys<R>) % 4 == 0, "cloud params must be word sized");
    const int* s = reinterpret_cast<const int*>(src);
    int* d = reinterpret_cast<int*>(&dst);
    for (int i = threadIdx.x; i < (int)(sizeof(CloudPhys<R>) / 4); i += blockDim.x) d[i] = s[i];
}

template <class R>
__device__ __forceinline__ R knife_cut_for(const CloudPhys<R>& P, double T, int step) {
    if (!(P.flags & F_KNIFE)) return R(0);
    double eta = knife_eta(P.knife_nknots, P.knife_step, P.knife_eta, (double)step);
    return (R)knife_cut_v2(eta, P.kB, T, P.mass);
}

// records accepted collisions of one cell: the atom ids of the pair and the direction n^
template <class R> struct TileCollisionLog {
    typedef typename V4T<R>::type R4;
    const R4* pos;   // the cell's staged positions (shared memory; atom id in the fourth lane)
    int2* ij;
    double* nv;
    int* count;
    int cap;
    int* err;
    template <class RR> __host__ __device__ void accept(uint32_t i, uint32_t j, RR nx, RR ny, RR nz) {
#if defined(__CUDA_ARCH__)
        const int slot = atomicAdd(count, 1);
        if (slot < cap) {
            ij[slot] = make_int2((int)lane_to_u32(pos[i].w), (int)lane_to_u32(pos[j].w));
            nv[3 * slot] = (double)nx;
            nv[3 * slot + 1] = (double)ny;
            nv[3 * slot + 2] = (double)nz;
        } else {
            atomicOr(err, EB_LOG_FULL);
        }
#endif
    }
};

// the collision record of a dense cell: atom ids read through the same permutation
template <class R> struct GatherCollisionLog {
    typedef typename V4T<R>::type R4;
    const R4* pos;
    const int* src;
    int capacity;
    int2* ij;
    double* nv;
    int* count;
    int cap;
    int* err;
    __device__ __forceinline__ int id(uint32_t i) const {
        const int s = src[i];
        return (s >= 0 && s < capacity) ? (int)lane_to_u32(pos[s].w) : -1;
    }
    template <class RR> __device__ void accept(uint32_t i, uint32_t j, RR nx, RR ny, RR nz) {
        const int slot = atomicAdd(count, 1);
        if (slot < cap) {
            ij[slot] = make_int2(id(i), id(j));
            nv[3 * slot] = (double)nx;
            nv[3 * slot + 1] = (double)ny;
            nv[3 * slot + 2] = (double)nz;
        } else {
            atomicOr(err, EB_LOG_FULL);
        }
    }
};

// 16-byte asynchronous global -> shared copies (cp.async, L2 only); a gather, unlike TMA
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::: "memory"); }

// an L2 prefetch of the line holding p (no register result, so nothing waits on it)
__device__ __forceinline__ void prefetch_l2(const void* p) { asm volatile("prefetch.global.L2 [%0];" ::"l"(p)); }
template <class R4> __device__ __forceinline__ void stage(R4* dst, const R4* src) {
#pragma unroll
    for (int o = 0; o < (int)sizeof(R4); o += 16)
        cp_async16(reinterpret_cast<char*>(dst) + o, reinterpret_cast<const char*>(src) + o);
}

__device__ __forceinline__ unsigned long long global_ns() {
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
// a look-back that sees no progress for this long gives up with EB_TIMEOUT instead of hanging
constexpr unsigned long long LB_TIMEOUT_NS = 1000000000ull;

// ---------------------------------------------------------------------------------------------
// dense_collide: the NTC collisions of the step's dense grid cells (more atoms than a tile stages
// beside a 512-atom tile), which step_pass leaves out.  One block per listed cell (a grid-stride
// loop over the list): the block gathers the cell's velocities through the sorted order's
// permutation into shared memory, one thread runs the same serial loop as a cell inside a tile --
// same collide_cell code, Philox words and order, so the same result bit for bit -- and the block
// writes them back.  A cell larger than the block's shared memory is gathered the same way into
// its own slots of the step's output velocity buffer instead (contiguous, in L2).  Launched before step_pass, which then gathers
// the collided velocities; cells are independent, so colliding them here or inside a tile is the
// same.  With no dense cell (the usual case) its blocks read the count and return.
// ---------------------------------------------------------------------------------------------
constexpr int DENSE_BLOCK = 512;
constexpr int DENSE_GRID = 148;
constexpr int DENSE_SMEM_BYTES = 200 * 1024;  // dynamic shared memory of a dense_collide block
template <class R>
__global__ void __launch_bounds__(DENSE_BLOCK) dense_collide(Args<R> A) {
    typedef typename V4T<R>::type R4;
    extern __shared__ __align__(16) unsigned char dense_smem[];
    R4* s_v = reinterpret_cast<R4*>(dense_smem);
    const int p = A.parity;
    const int nd = min(A.ctl->ndense[p], A.dense_cap);
    if (nd == 0) return;
    const int step = A.ctl->step[p];
    if (step % A.collide_every != 0) return;
    const int n_now = A.ctl->n[p];
    const int cap = (int)(DENSE_SMEM_BYTES / sizeof(R4));
    R4* const vel = const_cast<R4*>(A.vel_in);
    for (int i = blockIdx.x; i < nd; i += gridDim.x) {  // block-uniform: every value below is
        const int2 d = A.dense_list[i];
        const int c = d.x, k = d.y;
        if (c < 0 || c >= A.total_cells || k < 0 || k >= A.nclouds) {
            if (threadIdx.x == 0) atomicOr(&A.ctl->err, EB_INCONSISTENT);
            continue;
        }
        const CloudPhys<R>& P = A.clouds[k];
        if (!(P.flags & F_COLLIDE)) continue;
        const int c_beg = A.old_start[c], n = A.old_start[c + 1] - c_beg;
        if (c_beg < 0 || n < 0 || c_beg + n > n_now) {
            if (threadIdx.x == 0) atomicOr(&A.ctl->err, EB_INCONSISTENT);
            continue;
        }
        const int* src = A.src_in + c_beg;
        // the cell's velocities, contiguous: in shared memory when they fit, else in the cell's
        // slots of the buffer this step's step_pass writes later (free until then)
        R4* const stage_v = n <= cap ? s_v : A.vel_out + c_beg;
        constexpr int U = 4;  // gathers in flight per thread: the indices of four atoms, then their velocities
        for (int t0 = threadIdx.x; t0 < n; t0 += DENSE_BLOCK * U) {
            int s[U];
#pragma unroll
            for (int u = 0; u < U; ++u) s[u] = t0 + u * DENSE_BLOCK < n ? src[t0 + u * DENSE_BLOCK] : 0;
#pragma unroll
            for (int u = 0; u < U; ++u) {
                const int t = t0 + u * DENSE_BLOCK;
                if (t >= n) continue;
                if (s[u] >= 0 && s[u] < A.capacity) stage_v[t] = vel[s[u]];
                else atomicOr(&A.ctl->err, EB_INCONSISTENT);
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            R svm = A.sigvrmax[c];
            const uint32_t lc = (uint32_t)(c - P.cell_base);
            CollideResult<R> cr;
            if (A.clog_ij) {
                GatherCollisionLog<R> lg{A.pos_in, src, A.capacity, A.clog_ij, A.clog_n, A.clog_count, A.clog_cap,
                                         &A.ctl->err};
                cr = collide_cell<R, R4*, GatherCollisionLog<R>>(stage_v, n, svm, P, lc, (uint32_t)step, A.seed, &lg);
            } else {
                cr = collide_cell<R>(stage_v, n, svm, P, lc, (uint32_t)step, A.seed);
            }
            A.sigvrmax[c] = svm;
            CloudAccum* bucket = A.accum + k * ACC_BUCKETS + (i & (ACC_BUCKETS - 1));
            if (cr.accepted) atomicAdd(&bucket->coll, (unsigned long long)cr.accepted);
            if (cr.candidates) atomicAdd(&bucket->cand, (unsigned long long)cr.candidates);
            if (A.rec_cell_coll) A.rec_cell_coll[c] = make_int2(step, cr.accepted);
        }
        __syncthreads();
        for (int t0 = threadIdx.x; t0 < n; t0 += DENSE_BLOCK * U) {
            int s[U];
#pragma unroll
            for (int u = 0; u < U; ++u) s[u] = t0 + u * DENSE_BLOCK < n ? src[t0 + u * DENSE_BLOCK] : -1;
#pragma unroll
            for (int u = 0; u < U; ++u)
                if (s[u] >= 0 && s[u] < A.capacity) vel[s[u]] = stage_v[t0 + u * DENSE_BLOCK];
        }
        __syncthreads();  // the staging area is reused by the block's next cell
    }
}

// ---------------------------------------------------------------------------------------------
// step_pass: the timestep of one tile.
// The tile's positions and velocities are gathered through src into shared memory with
// asynchronous 16-byte copies issued all at once (CAP x 2 x R4), with each atom's storage index
// beside them; the cells collide from shared memory, then every atom moves, its spinor loaded
// through the kept index (only the motion phase reads it, so it takes no staging space and the
// tiles are larger); only the new state, the keys and the counters go back to global memory.
// ---------------------------------------------------------------------------------------------
// ONE: the run has a single cloud, whose parameters are read from the kernel parameter block
// (constant operands) instead of a shared-memory copy
template <class R, int BLOCK, int CAP, int MINB, bool ONE>
__global__ void __launch_bounds__(BLOCK, MINB) step_pass(const __grid_constant__ Args<R> A) {
    typedef typename V4T<R>::type R4;
    constexpr int PER = CAP / BLOCK;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    R4* s_pos = reinterpret_cast<R4*>(smem_raw);
    R4* s_vel = s_pos + CAP;
    int* s_src = reinterpret_cast<int*>(s_vel + CAP);  // storage index of each staged atom
    int* s_cell = s_src + CAP;
    uint16_t* s_head = reinterpret_cast<uint16_t*>(s_cell + CAP);  // first positions of cells to collide
    static_assert(CAP <= 65536, "head positions are 16-bit");
    static_assert(CAP <= (1 << KEY_RANK_BITS), "a stayer's rank (below CAP) must fit its key");
    constexpr int DENSE = dense_threshold(CAP);
    __shared__ CloudPhys<R> P_sh;
    const CloudPhys<R>& P = ONE ? A.one : P_sh;
    __shared__ StepAcc red[BLOCK / 32];
    __shared__ R s_cut;
    __shared__ int s_nhead;
    __shared__ int s_next_split;
    // the last run of cells in each 32-position chunk: its cell, its stayers, whether it spans the chunk
    constexpr int NCH = CAP / 32;
    __shared__ int s_tcell[NCH];
    __shared__ int s_tcnt[NCH];
    __shared__ int s_twhole[NCH];
    __shared__ LostAcc s_lost;

    const int p = A.parity;
    const int ntiles = A.ctl->ntiles[p];
    const int nprev = A.ctl->n[p];
    const int step = A.ctl->step[p];
    const int lane = threadIdx.x & 31;
    const bool collide_now = (step % A.collide_every) == 0;
    // MCWF phase of this step: bit 0 at the start of a collision period, bit 1 at its end
    const uint32_t mcwf_phase = (collide_now ? 1u : 0u) | (((step + 1) % A.collide_every) == 0 ? 2u : 0u);
    int cur_cloud = -1;
    if (threadIdx.x == 0) {
        LostAcc z = {};
        s_lost = z;  // ordered before first use by the barrier after the first load_cloud
    }

    // this warp's chunk of mover-list slots: the next free one and the chunk's end
    int mv_next = 0, mv_end = 0;
    // tiles in a grid-stride loop: the launch size only sets how many tiles run at once
    for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
        const int tb = A.tile_begin[b];
        const int te = A.tile_begin[b + 1];
        const int L = te - tb;
        const int cloud = A.tile_cloud[b];
        const int nsplit = b + 1 < ntiles ? A.tile_split[b + 1] : 0;  // with the bounds: one round trip
        if (cloud != cur_cloud) {  // block-uniform: the cloud's parameters and knife cut
            if (!ONE) load_cloud(P_sh, A.clouds + cloud);
            __syncthreads();
            if (threadIdx.x == 0) s_cut = knife_cut_for(P, A.cdyn[cloud].T_knife, step);
            __syncthreads();
            cur_cloud = cloud;
        }
        const bool box = (P.trap == TRAP_BOX);

        if (L > CAP || L < 0 || te > nprev) {
            // cannot stage this tile: every atom in it leaves the simulation (flagged), so the cell
            // counts stay consistent and every later kernel only touches indices it computed itself
            if (threadIdx.x == 0) atomicOr(&A.ctl->err, EB_CELL_FULL);
            for (int t = threadIdx.x; t < L && tb + t < nprev; t += BLOCK) {
                int s = A.src_in[tb + t];
                s = (s >= 0 && s < A.capacity) ? s : 0;
                const R4 q = A.pos_in[s];
                atomicAdd(&A.Lc[cell_of(P, q.x, q.y, q.z, box)], 1);
                A.keys[tb + t] = make_int2(-1, KIND_LOST);
            }
            if (threadIdx.x == 0) {
                A.tile_ovf[b] = 0;
                const int dropped = min(L, nprev - tb);
                if (!ONE && dropped > 0) atomicAdd(&A.cloud_lost[cloud], dropped);
            }
            if (!ONE) __syncthreads();  // the shared cloud parameters were read above; the next tile may replace them
            continue;
        }
        const R cut = s_cut;

        // phase 1: all storage indices, then all gathers in flight at once.  src values index the
        // buffer the previous step wrote, which held the atoms before that step's losses: they are
        // bounded by the capacity, not by the current count.
        int sidx[PER];
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int t = threadIdx.x + k * BLOCK;
            sidx[k] = t < L ? A.src_in[tb + t] : 0;
        }
#pragma unroll
        for (int k = 0; k < PER; ++k) {
            const int t = threadIdx.x + k * BLOCK;
            if (t < L) {
                int s = sidx[k];
                if (s < 0 || s >= A.capacity) {
                    atomicOr(&A.ctl->err, EB_INCONSISTENT);
                    s = 0;
                }
                stage(s_pos + t, A.pos_in + s);
                stage(s_vel + t, A.vel_in + s);
                s_src[t] = s;
                prefetch_l2(A.psi_in + s);  // read in the motion phase: an L2 hit by then
            }
        }
        if (threadIdx.x == 0) {
            s_nhead = 0;
            s_next_split = nsplit;  // whether the next tile begins inside this tile's last cell
        }
        // the next tile's storage indices into L2 (its first DRAM round trip), while the
        // gathers of this one are in flight
        {
            const int bn = b + gridDim.x;
            if (bn < ntiles && threadIdx.x < CAP / 32) {
                const int ntb = A.tile_begin[bn], nte = A.tile_begin[bn + 1];
                const int x = ntb + 32 * threadIdx.x;
                if (x < nte) prefetch_l2(A.src_in + x);
            }
        }
        // each thread's cell pass reads only the positions it staged itself: its own copies
        // suffice, the barrier after the pass publishes the cells and the staged tile
        cp_async_wait_all();
        for (int t = threadIdx.x; t < L; t += BLOCK) {
            const R4 q = s_pos[t];
            const int c = cell_of(P, q.x, q.y, q.z, box);
            s_cell[t] = c;
        }
        __syncthreads();
        const int c_first = L > 0 ? s_cell[0] : -1;
        const bool split = L > 0 && A.tile_split[b] != 0;

        StepAcc acc;
        zero_acc(acc);
        // phase 2: NTC collisions, one thread per grid cell that fits a tile (dense cells, which
        // dense_collide has collided, and the overflow cell are split across tiles).  The cells
        // holding two or more atoms are listed first, so that every lane takes a cell.
        if ((P.flags & F_COLLIDE) && collide_now) {
            for (int base = 0; base < L; base += BLOCK) {
                const int t = base + threadIdx.x;
                bool head = false;
                if (t + 1 < L) {
                    const int c = s_cell[t];
                    head = c != P.ovf_cell && (t == 0 || s_cell[t - 1] != c) && s_cell[t + 1] == c;
                }
                const unsigned hm = __ballot_sync(0xffffffffu, head);
                if (hm) {
                    int first = 0;
                    if (lane == 0) first = atomicAdd(&s_nhead, __popc(hm));
                    first = __shfl_sync(0xffffffffu, first, 0);
                    if (head) s_head[first + __popc(hm & ((1u << lane) - 1u))] = (uint16_t)t;
                }
            }
            __syncthreads();
            const int nhead = s_nhead;
            for (int h = threadIdx.x; h < nhead; h += BLOCK) {
                const int t = s_head[h];
                const int c = s_cell[t];
                // three independent loads in one round trip (c is a grid cell of this cloud)
                const int c_beg = A.old_start[c], c_end = A.old_start[c + 1];
                R svm = A.sigvrmax[c];
                const int n = c_end - c_beg;
                if (n > DENSE) continue;  // a dense cell: collided by dense_collide
                if (c_beg != tb + t || n > L - t) {  // cell not wholly inside this tile
                    atomicOr(&A.ctl->err, EB_INCONSISTENT);
                    continue;
                }
                if (n < 2) continue;
                CollideResult<R> cr;
                if (A.clog_ij) {
                    TileCollisionLog<R> lg{s_pos + t, A.clog_ij, A.clog_n, A.clog_count, A.clog_cap, &A.ctl->err};
                    cr = collide_cell<R, R4*, TileCollisionLog<R>>(s_vel + t, n, svm, P, (uint32_t)(c - P.cell_base),
                                                                   (uint32_t)step, A.seed, &lg);
                } else {
                    cr = collide_cell<R>(s_vel + t, n, svm, P, (uint32_t)(c - P.cell_base), (uint32_t)step,
                                             A.seed);
                }
                A.sigvrmax[c] = svm;
                acc.coll += (unsigned)cr.accepted;
                acc.cand += (unsigned)cr.candidates;
                if (A.rec_cell_coll) A.rec_cell_coll[c] = make_int2(step, cr.accepted);
            }
            __syncthreads();
        }

        // phase 3: move, spin, evaporate and classify every atom once
        for (int base = 0; base < L; base += BLOCK) {
            const int t = base + threadIdx.x;
            const bool valid = t < L;
            Atom<R> a;
            AtomOut<R> o;
            o.fate = FATE_ALIVE;
            o.cell = 0;
            bool stayer = false, mover = false;
            int c_old = 0;
            R4 q, v, s;
            if (valid) {
                s = A.psi_in[s_src[t]];
                q = s_pos[t];
                v = s_vel[t];
                a.x = q.x; a.y = q.y; a.z = q.z;
                a.vx = v.x; a.vy = v.y; a.vz = v.z;
                a.ur = s.x; a.ui = s.y; a.dr = s.z; a.di = s.w;
                a.flags = lane_to_u32(v.w);
                StepCtx sc;
                sc.id = lane_to_u32(q.w);
                sc.step = (uint32_t)step;
                sc.cloud = (uint32_t)P.cloud_id;
                sc.mcwf = mcwf_phase;
                sc.seed = A.seed;
                advance_atom(P, cut, a, o, sc);
                c_old = s_cell[t];
                const bool alive = (o.fate == FATE_ALIVE);
                stayer = alive && (o.cell == c_old);
                mover = alive && !stayer;
                if (!(o.v2 == o.v2)) atomicOr(&A.ctl->err, EB_NAN);
            }
            // stayers are ranked among the stayers of their cell in old order: cells are runs of
            // consecutive positions, so within this warp's 32 positions a stayer's rank is the number
            // of stayers since the start of its run; a run that continues from the previous chunk
            // gets that chunk's count after the block's next barrier
            const unsigned FULL = 0xffffffffu;
            const int cprev = __shfl_up_sync(FULL, c_old, 1);
            const unsigned vmask = __ballot_sync(FULL, valid);
            const unsigned hmask = __ballot_sync(FULL, valid && (lane == 0 || c_old != cprev));
            const unsigned smask = __ballot_sync(FULL, stayer);
            const int chunk = t >> 5;
            if (vmask) {
                const unsigned le = lane == 31 ? FULL : ((2u << lane) - 1u);
                const int run0 = 31 - __clz(hmask & le);
                const int tail0 = 31 - __clz(hmask);
                const int tcell = __shfl_sync(FULL, c_old, 31 - __clz(vmask));
                if (lane == 0) {
                    s_tcell[chunk] = tcell;
                    s_tcnt[chunk] = __popc(smask & (FULL << tail0));
                    s_twhole[chunk] = tail0 == 0 ? 1 : 0;
                }
                if (stayer) {
                    const int rank = __popc(smask & ((1u << lane) - 1u) & (FULL << run0));
                    const int cstart = t - lane;
                    const bool cont = run0 == 0 && cstart > 0 && (s_cell[cstart - 1] & 0x7fffffff) == c_old;
                    if (cont) {  // finished after the barrier
                        reinterpret_cast<int*>(s_pos + t)[0] = rank;
                        s_cell[t] = (int)((unsigned)c_old | 0x80000000u);
                    } else {
                        A.keys[tb + t] = stayer_key(split && c_old == c_first, b, c_old, rank, c_old == P.ovf_cell, cloud);
                    }
                }
            }
            // leavers of the old cell (movers and lost atoms): one fire-and-forget atomic each (a
            // warp pass rarely has two leavers of one cell, so aggregating them costs more than it saves)
            if (valid && !stayer) atomicAdd(&A.Lc[c_old], 1);
            // movers: a slot in the step's mover list from the warp's chunk (the chunk's last slots, then
            // a new chunk when this pass's movers do not fit), and one more incoming atom for the
            // target cell, counted without waiting for the result (permute_pass hands out the
            // cells' incoming slots)
            const unsigned mm = __ballot_sync(0xffffffffu, mover);
            int slot = 0;
            if (mm) {
                const int need = __popc(mm);
                const int rank = __popc(mm & ((1u << lane) - 1u));
                const int left = mv_end - mv_next;
                if (need <= left) {
                    slot = mv_next + rank;
                    mv_next += need;
                } else {
                    int nb = 0;
                    if (lane == 0) nb = atomicAdd(&A.ctl->movers[p], MV_CHUNK);
                    nb = __shfl_sync(0xffffffffu, nb, 0);
                    slot = rank < left ? mv_next + rank : nb + (rank - left);
                    mv_next = nb + (need - left);
                    mv_end = nb + MV_CHUNK;
                }
            }
            if (mover) {
                atomicAdd(&A.Ic[o.cell], 1);
                if (slot < A.mrec_cap)
                    A.mrec[slot] = make_int4(o.cell, tb + t, 0, cloud | (o.cell == P.ovf_cell ? MREC_OVF_CELL : 0));
                else
                    atomicOr(&A.ctl->err, EB_CAPACITY);
            }
            if (valid) {
                const int j = tb + t;
                if (stayer || mover) {
                    R4 qo, vo, so;
                    qo.x = a.x; qo.y = a.y; qo.z = a.z; qo.w = q.w;
                    vo.x = a.vx; vo.y = a.vy; vo.z = a.vz; vo.w = lane_from_u32(a.flags, R(0));
                    so.x = a.ur; so.y = a.ui; so.z = a.dr; so.w = a.di;
                    A.pos_out[j] = qo;
                    A.vel_out[j] = vo;
                    A.psi_out[j] = so;
                    acc.n_alive += 1u;
                    acc.sum_v2 += fx_from_magnitude(o.v2);  // v^2 >= 0: fx_from without the sign
                    acc.sum_B += fx_from(o.absB);
                    if (!stayer) A.keys[j] = make_int2(slot, KIND_MOVE);
                } else {
                    add_limbs(s_lost.ev2, fx_from(o.v2));
                    add_limbs(s_lost.eB, fx_from(o.absB));
                    atomicAdd(o.fate == FATE_MAJORANA ? &s_lost.n_maj : &s_lost.n_knife, 1ull);
                    A.keys[j] = make_int2(-1, KIND_LOST);
                    const unsigned id = lane_to_u32(q.w);
                    if (A.rec_evap_pos && id < (unsigned)P.id_cap) {  // the snapshot record of a lost atom
                        R4 ep, ev;
                        ep.x = a.x; ep.y = a.y; ep.z = a.z; ep.w = lane_from_u32((uint32_t)step, R(0));
                        ev.x = a.vx; ev.y = a.vy; ev.z = a.vz; ev.w = lane_from_u32((uint32_t)o.fate, R(0));
                        A.rec_evap_pos[P.id_base + id] = ep;
                        A.rec_evap_vel[P.id_base + id] = ev;
                    }
                }
            }
        }
        TilePartial tot;
        block_reduce_acc<BLOCK>(acc, red, tot);  // its barrier also orders the chunk records and s_lost
        if (threadIdx.x == 0) {
            CloudAccum* bucket = A.accum + cloud * ACC_BUCKETS + (b & (ACC_BUCKETS - 1));
            // when the next tile begins inside this tile's last cell (split): that cell's stayers here,
            // from the chunk records of its run (counted for the ranks of its stayers there), and
            // whether this tile lies wholly inside it
            int cont = 0;
            bool whole = false;
            if (s_next_split && L > 0) {
                const int lc = (L - 1) >> 5;
                const int c_last = s_tcell[lc];
                for (int qq = lc; qq >= 0 && s_tcell[qq] == c_last; --qq) {
                    cont += s_tcnt[qq];
                    if (!s_twhole[qq]) break;
                }
                whole = split && c_last == c_first;
            }
            A.tile_ovf[b] = cont | (whole ? TILE_WHOLE : 0);
            if (split) A.tile_cell[b] = c_first;
            if (cont > 0 || split) {  // ovf_carries scans the tiles from the lowest to the highest listed
                const int i = atomicAdd(&A.ctl->novf[p], 1);
                if (i < A.max_tiles) A.ovf_list[i] = b;
            }
            accum_tile(bucket, tot);
            const unsigned long long nlost = s_lost.n_maj + s_lost.n_knife;
            if (!ONE && nlost) atomicAdd(&A.cloud_lost[cloud], (int)nlost);  // one cloud: its scan needs none
            accum_lost(bucket, s_lost);
        }
        // stayers whose cell run began in an earlier chunk: add the stayers of that run there
        for (int t = threadIdx.x; t < L; t += BLOCK) {
            const int cm = s_cell[t];
            if (cm >= 0) continue;
            const int c = cm & 0x7fffffff;
            int rank = reinterpret_cast<const int*>(s_pos + t)[0];
            for (int qq = (t >> 5) - 1; qq >= 0 && s_tcell[qq] == c; --qq) {
                rank += s_tcnt[qq];
                if (!s_twhole[qq]) break;
            }
            A.keys[tb + t] = stayer_key(split && c == c_first, b, c, rank, c == P.ovf_cell, cloud);
        }
        __syncthreads();  // the staging arrays, red and s_lost are reused by the next tile
    }
    for (int i = mv_next + lane; i < mv_end; i += 32)  // the last chunk's unused slots
        if (i < A.mrec_cap) A.mrec[i] = make_int4(-1, -1, -1, -1);
}

// ---------------------------------------------------------------------------------------------
// Tile starts of the coming step, written where the atoms are placed (permute_pass, mover_rank,
// and init_tiles after a full sort).  The nominal starts S + j*T of cloud k (S its first sorted
// position, T the coming nominal size) that fall inside a grid cell [st, e) snap to the cell's end,
// except one exactly at st; a split cell -- the overflow cell, which never collides, or a dense
// cell, which dense_collide collides -- begins a tile at each nominal start inside it.
// ---------------------------------------------------------------------------------------------
// every tile start in the non-empty cell [st, e) of cloud k
template <class R>
__device__ void cell_tile_starts(const Args<R>& A, int k, int st, int e, bool ovf) {
    const int q = 1 - A.parity;
    const int S = A.cdyn[k].start[q], toff = A.cdyn[k].tile_off[q];
    const int T = A.ctl->tile_T[q];
    if (T <= 0 || st < S) {
        atomicOr(&A.ctl->err, EB_INCONSISTENT);
        return;
    }
    for (int j = (st - S + T - 1) / T; S + j * T < e; ++j) {
        const int pnom = S + j * T;
        const int tbeg = pnom == st ? st : (ovf ? pnom : e);
        const int ti = toff + j;
        if (ti < A.max_tiles) {
            A.tile_begin_next[ti] = tbeg;
            A.tile_cloud_next[ti] = k;
            A.tile_split_next[ti] = (tbeg != st && tbeg != e) ? 1 : 0;
        }
    }
}

// lists grid cell c of cloud k, dense in the coming step, for that step's dense_collide (called once per
// dense cell: by the atom placed at its first position, or by init_tiles after a full sort)
template <class R>
__device__ __forceinline__ void list_dense(const Args<R>& A, int c, int k) {
    const int i = atomicAdd(&A.ctl->ndense[1 - A.parity], 1);
    if (i < A.dense_cap) A.dense_list[i] = make_int2(c, k);
    else atomicOr(&A.ctl->err, EB_CAPACITY);
}

// the tile start at position x of a split cell of cloud k (the cell begins at st), if x is a nominal start
template <class R>
__device__ __forceinline__ void split_tile_start(const Args<R>& A, int k, int st, int x) {
    const int q = 1 - A.parity;
    const int S = A.cdyn[k].start[q];
    const int T = A.ctl->tile_T[q];
    const int r = x - S;
    if (T <= 0 || r < 0 || r % T != 0) return;
    const int ti = A.cdyn[k].tile_off[q] + r / T;
    if (ti < A.max_tiles) {
        A.tile_begin_next[ti] = x;
        A.tile_cloud_next[ti] = k;
        A.tile_split_next[ti] = x != st ? 1 : 0;
    }
}

// ---------------------------------------------------------------------------------------------
// permute_pass: the stayers' part of the next step's gather permutation.  A stayer of cell c with
// rank r goes to new_start[c] + r (+ the stayers of its split cell in the cell's earlier tiles for
// KIND_OVF); src_out[dest] = its position in the buffer step_pass wrote.  Unless scan_cells built
// the coming tiling, the stayer placed at a grid cell's first position writes the cell's tile
// starts; every stayer of a split cell (the overflow cell, or a cell that will be dense) checks its
// own position.  Movers are placed by
// mover_rank, after this kernel has listed each cell's incoming movers.  Flat streams over the
// keys and the mover records, no shared memory and no barriers.
// ---------------------------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) permute_pass(Args<R> A) {
    const int p = A.parity;
    const int n = A.ctl->n[p];
    const int ntiles = A.ctl->ntiles[p];
    const bool tiles = A.ctl->tiles_built[1 - p] == 0;  // the coming tiling is built here
    const int dense = dense_threshold(A.tile_cap);     // larger cells are split like the overflow cell
    // four consecutive positions per thread and pass: two 16-byte key loads, then the cell
    // starts of all four, then the stores (the loads of one pass are independent)
    constexpr int G = 4;
    for (int j0 = (blockIdx.x * 256 + threadIdx.x) * G; j0 < n; j0 += gridDim.x * 256 * G) {
        int2 key[G];
        if (j0 + G <= n) {
            const int4 a = reinterpret_cast<const int4*>(A.keys + j0)[0];
            const int4 b = reinterpret_cast<const int4*>(A.keys + j0)[1];
            key[0] = make_int2(a.x, a.y); key[1] = make_int2(a.z, a.w);
            key[2] = make_int2(b.x, b.y); key[3] = make_int2(b.z, b.w);
        } else {
#pragma unroll
            for (int i = 0; i < G; ++i) key[i] = j0 + i < n ? A.keys[j0 + i] : make_int2(-1, KIND_LOST);
        }
        int c[G], base[G];
        bool ok[G];
#pragma unroll
        for (int i = 0; i < G; ++i) {
            const int kind = key[i].y & 3;
            ok[i] = kind == KIND_STAY || kind == KIND_OVF;
            c[i] = key[i].x;
            base[i] = 0;
            if (kind == KIND_OVF) {
                const int b = key[i].x;
                if (b < 0 || b >= ntiles) {
                    atomicOr(&A.ctl->err, EB_INCONSISTENT);
                    ok[i] = false;
                    continue;
                }
                c[i] = A.tile_cell[b];  // the split cell the tile begins inside
                base[i] = A.tile_ovf_carry[b];
            }
            if (ok[i] && (c[i] < 0 || c[i] >= A.total_cells)) {
                atomicOr(&A.ctl->err, EB_INCONSISTENT);
                ok[i] = false;
            }
        }
        int lo[G], hi[G];
#pragma unroll
        for (int i = 0; i < G; ++i) {
            lo[i] = ok[i] ? A.new_start[c[i]] : 0;
            hi[i] = ok[i] ? A.new_start[c[i] + 1] : 0;
        }
#pragma unroll
        for (int i = 0; i < G; ++i) {
            if (!ok[i]) continue;
            const int r = base[i] + ((key[i].y >> KEY_RANK_SHIFT) & KEY_RANK_MASK);
            const int dest = lo[i] + r;
            if (dest >= lo[i] && dest < hi[i] && dest < A.capacity) {
                A.src_out[dest] = j0 + i;
                const int kcl = key[i].y >> KEY_CLOUD_SHIFT;  // the cell's cloud
                const bool ovf = (key[i].y & KEY_OVF_CELL) != 0;
                const bool dns = !ovf && hi[i] - lo[i] > dense;
                if (dns && r == 0) list_dense(A, c[i], kcl);
                if (tiles) {
                    if (ovf || dns) split_tile_start(A, kcl, lo[i], dest);
                    else if (r == 0) cell_tile_starts(A, kcl, lo[i], hi[i], false);
                }
            } else {
                atomicOr(&A.ctl->err, EB_INCONSISTENT);
            }
        }
    }
    // incoming movers: each takes a slot in its cell's incoming list (the scan cleared the cell's
    // incoming count, which now counts the slots handed out) and writes its old position there
    const int m = min(A.ctl->movers[p], A.mrec_cap);
    for (int i = blockIdx.x * 256 + threadIdx.x; i < m; i += gridDim.x * 256) {
        const int4 r = A.mrec[i];
        if (r.x < 0) continue;  // an unused slot of a warp's chunk
        const int slot = A.mover_base[r.x] + atomicAdd(&A.Ic[r.x], 1);
        if (slot >= 0 && slot < A.new_start[r.x + 1] && slot < A.capacity) A.in_list[slot] = r.y;
        else atomicOr(&A.ctl->err, EB_INCONSISTENT);
    }
}

// ---------------------------------------------------------------------------------------------
// The cell scan of a step, in one pass (scan_cells).  Each scan block covers <= CB * CELL_ITEMS cells of
// one cloud; the count of cell c after the step is (old_start[c+1] - old_start[c]) - L[c] + I[c].
// A block takes its scan block from a ticket (scan blocks are handed out in the order the blocks
// start), publishes its sum, and finds its offset by looking back over the descriptors of the scan
// blocks before it: it only ever waits on blocks that started before it, and every wait is
// bounded in time.  A block covers the cells [c0, c1) of one cloud; a cloud whose cells start off
// a 4-cell boundary has a short first block up to it, so that its other blocks load and store
// 16-byte vectors.
// ---------------------------------------------------------------------------------------------
constexpr int SCAN_BLOCK = 256;
constexpr int SCAN_ITEMS = 8;  // items per thread of the generic scans (gscan_*)
constexpr int SCAN_CHUNK = SCAN_BLOCK * SCAN_ITEMS;
#ifndef DSMC_LB_STRIDE
#define DSMC_LB_STRIDE 32
#endif
// scan_cells block: CELL_BLOCK threads (four blocks per SM at 64 registers, so that one block's
// loads overlap another's look-back and barriers), ITEMS cells each: 16 on grids that give every SM
// two blocks or more at that size, else 8 (more, shorter blocks for a small grid's short step)
constexpr int CELL_BLOCK = 256;
inline int cell_items_for(int total_cells) { return total_cells >= 2 * 148 * CELL_BLOCK * 16 ? 16 : 8; }
// descriptors lie LB_STRIDE words apart (one per 256 bytes), so that the look-back reads of all
// blocks spread over the L2 slices instead of queueing on the few that hold a dense array
constexpr int LB_STRIDE = DSMC_LB_STRIDE;

// blocks of a physics-step scan_cells launch ahead of its scan blocks: one for the overflow-cell
// carries, then one per cb / 32 clouds for the clouds' step totals
inline int scan_extra_blocks(int nclouds, int cb) { return 1 + (nclouds + cb / 32 - 1) / (cb / 32); }

// descriptor of a scan block, one 64-bit word: (epoch << 34) | (status << 32) | value, where the
// epoch numbers the scan launch that wrote it (a word left by an earlier launch reads as not ready)
// and the value is the block's sum (LB_AGG) or its inclusive prefix (LB_INC)
enum : unsigned { LB_NONE = 0, LB_AGG = 1, LB_INC = 2 };
constexpr unsigned LB_EPOCH_MASK = 0x3fffffffu;

__device__ __forceinline__ unsigned long long lb_word(unsigned epoch, unsigned status, unsigned v) {
    return ((unsigned long long)(epoch & LB_EPOCH_MASK) << 34) | ((unsigned long long)status << 32) | v;
}
__device__ __forceinline__ unsigned lb_status(unsigned long long w, unsigned epoch) {
    return (unsigned)(w >> 34) == (epoch & LB_EPOCH_MASK) ? (unsigned)(w >> 32) & 3u : LB_NONE;
}
// the descriptor word carries all its data, so device-scope relaxed accesses suffice
__device__ __forceinline__ void lb_store(unsigned long long* desc, int b, unsigned long long w) {
    unsigned long long* p = desc + (size_t)b * LB_STRIDE;
    asm volatile("st.relaxed.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(w) : "memory");
}
__device__ __forceinline__ unsigned long long lb_load(const unsigned long long* desc, int b) {
    const unsigned long long* p = desc + (size_t)b * LB_STRIDE;
    unsigned long long w;
    asm volatile("ld.relaxed.gpu.global.u64 %0, [%1];" : "=l"(w) : "l"(p) : "memory");
    return w;
}

// Exclusive prefix of scan block blk (one full warp; the result is the same in every lane).  The
// warp reads the LB_WINDOW descriptors before it (lane l holds distances 8l .. 8l+7, nearest
// first) and adds the values up to the nearest inclusive prefix once all of them are published;
// with none in the window it adds them all and moves on.
constexpr int LB_PER_LANE = 8;
constexpr int LB_WINDOW = 32 * LB_PER_LANE;
__device__ unsigned lb_exclusive(const unsigned long long* desc, int blk, unsigned epoch, int* err) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    unsigned excl = 0;
    int base = blk - 1;
    const unsigned long long t0 = global_ns();
    while (base >= 0) {
        unsigned v[LB_PER_LANE];
        unsigned incm = 0, pendm = 0;
#pragma unroll
        for (int u = 0; u < LB_PER_LANE; ++u) {
            const int i = base - lane * LB_PER_LANE - u;
            const unsigned long long w = i >= 0 ? lb_load(desc, i) : lb_word(epoch, LB_INC, 0u);
            const unsigned st = lb_status(w, epoch);
            v[u] = (unsigned)w;
            incm |= (st == LB_INC ? 1u : 0u) << u;
            pendm |= (st == LB_NONE ? 1u : 0u) << u;
        }
        const unsigned inc = __ballot_sync(FULL, incm != 0);
        const int near = inc ? __ffs(inc) - 1 : 32;  // nearest lane holding an inclusive prefix
        // positions of this lane that count: all before the nearest lane, up to its first inclusive
        const unsigned use = lane < near ? (1u << LB_PER_LANE) - 1u
                                         : (lane == near ? ((incm & (0u - incm)) << 1) - 1u : 0u);
        if (!__any_sync(FULL, (pendm & use) != 0)) {
            unsigned sum = 0;
#pragma unroll
            for (int u = 0; u < LB_PER_LANE; ++u) sum += ((use >> u) & 1u) ? v[u] : 0u;
            excl += __reduce_add_sync(FULL, sum);
            if (inc) break;
            base -= LB_WINDOW;
            continue;
        }
        const bool late = __shfl_sync(FULL, global_ns() - t0 > LB_TIMEOUT_NS ? 1 : 0, 0) != 0;
        if (late) {
            if (lane == 0) atomicOr(err, EB_TIMEOUT);
            break;
        }
        __nanosleep(32);
    }
    return excl;
}

// Step totals of cloud k from its buckets (one warp; the buckets are cleared), the knife
// temperature of the coming step, and on cloud 0 the step counter of the coming step.
template <class R, bool INIT>
__device__ __forceinline__ void finalize_cloud(const Args<R>& A, int k, int lane) {
    static_assert(ACC_BUCKETS <= 32, "one lane per bucket");
    const int p = A.parity;
    CloudDyn& d = A.cdyn[k];
    TilePartial acc;
    zero_partial(acc);
    if (lane < ACC_BUCKETS) {
        CloudAccum& g = A.accum[k * ACC_BUCKETS + lane];
        acc.sum_v2 = from_limbs(g.v2);
        acc.sum_B = from_limbs(g.B);
        acc.evap_v2 = from_limbs(g.ev2);
        acc.evap_B = from_limbs(g.eB);
        acc.n_alive = (long long)g.n_alive;
        acc.n_maj = (long long)g.n_maj;
        acc.n_knife = (long long)g.n_knife;
        acc.coll = (long long)g.coll;
        acc.cand = (long long)g.cand;
        CloudAccum z = {};
        g = z;  // cleared for the next step
    }
    acc.sum_v2 = warp_sum_i128(acc.sum_v2);
    acc.sum_B = warp_sum_i128(acc.sum_B);
    acc.evap_v2 = warp_sum_i128(acc.evap_v2);
    acc.evap_B = warp_sum_i128(acc.evap_B);
    acc.n_alive = warp_sum_ll(acc.n_alive);
    acc.n_maj = warp_sum_ll(acc.n_maj);
    acc.n_knife = warp_sum_ll(acc.n_knife);
    acc.coll = warp_sum_ll(acc.coll);
    acc.cand = warp_sum_ll(acc.cand);
    if (lane == 0) {
        const CloudPhys<R>& P = A.clouds[k];
        CloudDiagDev& g = A.cdiag[k];
        const int step_now = A.ctl->step[p];
        if (INIT) {
            g.step = step_now;
            g.cum_evap = 0; g.cum_maj = 0; g.cum_knife = 0; g.cum_coll = 0; g.cum_cand = 0;
            g.cum_evap_v2 = 0; g.cum_evap_B = 0; g.cum_atom_steps = 0;
        } else {
            g.step = step_now + 1;
            g.cum_evap += acc.n_maj + acc.n_knife;
            g.cum_maj += acc.n_maj;
            g.cum_knife += acc.n_knife;
            g.cum_coll += acc.coll;
            g.cum_cand += acc.cand;
            g.cum_evap_v2 += acc.evap_v2;
            g.cum_evap_B += acc.evap_B;
            g.cum_atom_steps += acc.n_alive + acc.n_maj + acc.n_knife;
        }
        g.n_alive = acc.n_alive;
        g.sum_v2 = acc.sum_v2;
        g.sum_B = acc.sum_B;
        g.err = A.ctl->err;
        d.T_knife = knife_temperature(P.mass, P.kB, P.T0, (P.flags & F_KNIFE_FIXED_T) != 0, acc.sum_v2,
                                      acc.n_alive);
        if (k == 0 && !INIT) {
            A.ctl->step[1 - p] = step_now + 1;
            if (A.clog_off) {
                const int rel = step_now + 1 - A.clog_step0;
                const int cnt = *A.clog_count;
                if (rel >= 1 && rel <= A.clog_steps) A.clog_off[rel] = cnt < A.clog_cap ? cnt : A.clog_cap;
            }
        }
    }
}

// diagnostics of the sorted state after initialisation (one warp per cloud)
template <class R, bool INIT>
__global__ void __launch_bounds__(32) finalize(Args<R> A) {
    finalize_cloud<R, INIT>(A, blockIdx.x, threadIdx.x);
}

// Top level of the cell scan, run by the last scan_cells block to finish: per-cloud counts, starts
// and tile offsets of the coming step (from the blocks' inclusive prefixes), the coming step's
// counters and nominal tile size, and the reset of the scan's ticket for the next launch.
template <class R, int BLOCK>
__device__ void scan_top_block(const Args<R>& A, unsigned epoch) {
    __shared__ uint32_t wsum[32];
    __shared__ int s_tcarry;
    const int q = 1 - A.parity;
    int total = (int)(unsigned)lb_load(A.scan_desc, A.nscan_blocks - 1);
    if (total < 0 || total > A.capacity) {  // only after an inconsistent step: keep every later index in range
        if (threadIdx.x == 0) atomicOr(&A.ctl->err, EB_INCONSISTENT);
        total = total < 0 ? 0 : A.capacity;
    }
    // the coming tiling's nominal size: the preferred size, or less where a cell holds so many
    // atoms that a tile snapped to cell boundaries could outgrow the staging capacity
    const int mc = __ldcg(&A.ctl->max_cell);
    int Tn = A.tile_nominal;
    if (A.tile_fill > 0 && A.tile_pass > 0) {
        // default size for a small run: the largest tile just under a whole number of block
        // passes that still gives every resident block a tile (a 1e4-atom cloud then runs 240-atom
        // tiles on 40 blocks instead of 1008-atom tiles on 10)
        const int per_block = total / A.tile_fill;
        const int passes = max(1, min((per_block + 16) / A.tile_pass, (Tn + 16) / A.tile_pass));
        Tn = min(Tn, passes * A.tile_pass - 16);
    }
    const int T = max(min(Tn, A.tile_cap + 1 - mc), MIN_TILE);
    // per-cloud counts, starts, tile offsets (clouds in chunks of BLOCK; one cloud holds them all)
    if (threadIdx.x == 0) s_tcarry = 0;
    if (A.nclouds == 1 && threadIdx.x == 0) {
        CloudDyn& d = A.cdyn[0];
        d.n[q] = total;
        d.start[q] = 0;
        d.ntiles[q] = (total + T - 1) / T;
        d.tile_off[q] = 0;
        s_tcarry = d.ntiles[q];
    }
    __syncthreads();
    for (int base = 0; A.nclouds > 1 && base < A.nclouds; base += BLOCK) {
        const int k = base + threadIdx.x;
        int n = 0, st = 0, nt = 0;
        if (k < A.nclouds) {
            const int fb = A.cloud_first_blk[k], lb = A.cloud_first_blk[k + 1] - 1;
            st = fb > 0 ? (int)(unsigned)lb_load(A.scan_desc, fb - 1) : 0;
            n = (int)(unsigned)lb_load(A.scan_desc, lb) - st;
            nt = (n + T - 1) / T;
        }
        uint32_t tot;
        const uint32_t ex = block_excl_scan_u32<BLOCK>((uint32_t)nt, wsum, tot);
        if (k < A.nclouds) {
            CloudDyn& d = A.cdyn[k];
            d.n[q] = n;
            d.start[q] = st;
            d.ntiles[q] = nt;
            d.tile_off[q] = (int)ex + s_tcarry;
        }
        __syncthreads();
        if (threadIdx.x == 0) s_tcarry += (int)tot;
        __syncthreads();
    }
    const int ntiles_next = s_tcarry;
    if (threadIdx.x == 0) {
        A.ctl->n[q] = total;
        A.ctl->ntiles[q] = ntiles_next > A.max_tiles ? A.max_tiles : ntiles_next;
        if (ntiles_next > A.max_tiles) atomicOr(&A.ctl->err, EB_TILE_OVERFLOW);
        A.new_start[A.total_cells] = total;
        A.tile_begin_next[ntiles_next <= A.max_tiles ? ntiles_next : A.max_tiles] = total;
        A.ctl->movers[q] = 0;
        A.ctl->novf[q] = 0;
        A.ctl->ndense[q] = 0;  // the coming step's dense cells are listed where its atoms are placed
        A.ctl->tiles_built[q] = (A.nclouds == 1 && !A.init_mode && T == A.ctl->tile_T[A.parity]) ? 1 : 0;
        A.ctl->tile_T[q] = T;
        A.ctl->max_cell = 0;
        A.ctl->scan_ticket = 0;
        A.ctl->scan_epoch = epoch + 1;
    }
    for (int k = threadIdx.x; k < A.nclouds; k += BLOCK) A.cloud_lost[k] = 0;  // read by this scan's cloud heads
}

// Stayers of split cells (overflow and dense cells), run by one block of a physics-step scan_cells
// launch beside the scan.  A stayer in a tile that begins inside its cell (a KIND_OVF key) is
// ranked after the cell's stayers in the cell's earlier tiles; that carry is, per tile b,
//   carry[b + 1] = cnt[b] + (whole[b] ? carry[b] : 0)
// with cnt[b] the stayers of tile b's last cell when that cell continues into tile b + 1, and
// whole[b] when tile b lies inside it.  An affine recurrence: the block scans it over the tiles
// from the lowest to the highest listed one (every split tile and every tile with cnt > 0 is
// listed, so the lowest listed tile has carry 0 and every carry a KIND_OVF key needs is in range).
template <class R, int BLOCK>
__device__ void ovf_carries(const Args<R>& A) {
    constexpr int NW = BLOCK / 32;
    __shared__ int s_lo, s_hi, s_x;
    __shared__ int wa[NW], wc[NW], wx[NW];
    const int p = A.parity;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    if (threadIdx.x == 0) {
        s_lo = 0x7fffffff;
        s_hi = -1;
        s_x = 0;
    }
    __syncthreads();
    const int m = min(A.ctl->novf[p], A.max_tiles);
    for (int i = threadIdx.x; i < m; i += BLOCK) {
        const int b = A.ovf_list[i];
        atomicMin(&s_lo, b);
        atomicMax(&s_hi, b);
    }
    __syncthreads();
    const int lo = s_lo, hi = s_hi;
    constexpr int IT = 16;
    for (int base = lo; base <= hi; base += BLOCK * IT) {
        const int i0 = base + threadIdx.x * IT;
        int cnt[IT];
        bool wh[IT];
        // this thread's tiles as one map x -> (a ? x : 0) + c (beyond hi: the identity)
        bool a = true;
        int c = 0;
#pragma unroll
        for (int k = 0; k < IT; ++k) {
            const int v = (i0 + k <= hi) ? A.tile_ovf[i0 + k] : TILE_WHOLE;
            cnt[k] = v & (TILE_WHOLE - 1);
            wh[k] = (v & TILE_WHOLE) != 0;
            c = (wh[k] ? c : 0) + cnt[k];
            a = a && wh[k];
        }
        // inclusive scan of the maps over the warp (later after earlier), then the exclusive one
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int ap = __shfl_up_sync(0xffffffffu, a ? 1 : 0, off);
            const int cp = __shfl_up_sync(0xffffffffu, c, off);
            if (lane >= off) {
                c = (a ? cp : 0) + c;
                a = a && ap != 0;
            }
        }
        int ae = __shfl_up_sync(0xffffffffu, a ? 1 : 0, 1);
        int ce = __shfl_up_sync(0xffffffffu, c, 1);
        if (lane == 0) {
            ae = 1;
            ce = 0;
        }
        if (lane == 31) {
            wa[warp] = a ? 1 : 0;
            wc[warp] = c;
        }
        __syncthreads();
        if (threadIdx.x == 0) {  // the carry entering each warp's first tile, and the next chunk's
            int x = s_x;
            for (int w = 0; w < NW; ++w) {
                wx[w] = x;
                x = (wa[w] ? x : 0) + wc[w];
            }
            s_x = x;
        }
        __syncthreads();
        int x = (ae ? wx[warp] : 0) + ce;
#pragma unroll
        for (int k = 0; k < IT; ++k) {
            if (i0 + k <= hi) A.tile_ovf_carry[i0 + k] = x;
            x = (wh[k] ? x : 0) + cnt[k];
        }
        __syncthreads();  // wa / wc / wx are rewritten by the next chunk
    }
}

// The cell scan of a step: new start[], the movers' base slots, cleared leaver / incoming counters,
// the largest grid-cell count, and (last block) the top level.  In a physics step the launch puts
// scan_extra_blocks(nclouds, CB) blocks ahead of the scan blocks: the overflow-cell carries, then the
// clouds' step totals, one warp per cloud; after a full sort it carries the scan blocks alone.
// MULTI: the handle holds more than one cloud (each cloud's look-back chain starts at its first block)
template <class R, int CB, int CELL_ITEMS, bool MULTI>
__global__ void __launch_bounds__(CB, 1024 / CB) scan_cells(Args<R> A) {
    constexpr int CELL_CHUNK = CB * CELL_ITEMS;
    __shared__ uint32_t wsum[32];
    __shared__ int s_blk, s_last, s_max;
    __shared__ unsigned s_excl;
    __shared__ int s_ovf_st, s_ovf_end;  // the overflow cell's range, when this block holds it
    const int nextra = (int)gridDim.x - A.nscan_blocks;
    if ((int)blockIdx.x < nextra) {
        if (A.init_mode) return;
        if (blockIdx.x == 0) {
            ovf_carries<R, CB>(A);
        } else {
            const int k = (blockIdx.x - 1) * (CB / 32) + (threadIdx.x >> 5);
            if (k < A.nclouds) finalize_cloud<R, false>(A, k, threadIdx.x & 31);
        }
        return;
    }
    const int lane = threadIdx.x & 31;
    const bool spec = A.nclouds == 1 && !A.init_mode;
    const unsigned epoch = *reinterpret_cast<volatile unsigned*>(&A.ctl->scan_epoch);
    if (threadIdx.x == 0) {
        s_blk = atomicAdd(&A.ctl->scan_ticket, 1);
        s_max = 0;
        s_ovf_st = 0;
        s_ovf_end = 0;
    }
    __syncthreads();
    const int blk = s_blk;
    if (blk < A.nscan_blocks) {
        const int4 hb = A.scan_blk[blk];
        const int head_blk = MULTI ? A.cloud_first_blk[hb.x] : 0;  // used at the look-back: loaded with the cells
        const int c0 = hb.y, cend = hb.z, c1 = hb.w;  // this block's cells [c0, c1) of a cloud ending at cend
        const int cb = c0 + threadIdx.x * CELL_ITEMS;
        // a block of CELL_CHUNK cells from a 16-byte boundary: vector loads and stores
        const bool whole = (c0 & 3) == 0 && c1 - c0 == CELL_CHUNK;
        constexpr int NV = CELL_ITEMS / 4;
        int cnt[CELL_ITEMS], in[CELL_ITEMS];
        unsigned lmask = 0, imask = 0;  // cells with leavers / incoming movers (counters to clear)
        if (whole) {
            int sv[CELL_ITEMS + 1];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const int4 t = *reinterpret_cast<const int4*>(A.old_start + cb + 4 * v);
                sv[4 * v] = t.x; sv[4 * v + 1] = t.y; sv[4 * v + 2] = t.z; sv[4 * v + 3] = t.w;
            }
            sv[CELL_ITEMS] = A.old_start[cb + CELL_ITEMS];
#pragma unroll
            for (int v = 0; v < NV; ++v) {
                const int4 l = *reinterpret_cast<const int4*>(A.Lc + cb + 4 * v);
                const int4 m = *reinterpret_cast<const int4*>(A.Ic + cb + 4 * v);
                const int lv[4] = {l.x, l.y, l.z, l.w};
                const int iv[4] = {m.x, m.y, m.z, m.w};
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = 4 * v + u;
                    in[k] = iv[u];
                    cnt[k] = sv[k + 1] - sv[k] - lv[u] + iv[u];
                    lmask |= (lv[u] != 0 ? 1u : 0u) << k;
                    imask |= (iv[u] != 0 ? 1u : 0u) << k;
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < CELL_ITEMS; ++k) {
                const int c = cb + k;
                const bool ok = c < c1;
                const int lv = ok ? A.Lc[c] : 0;
                in[k] = ok ? A.Ic[c] : 0;
                cnt[k] = ok ? A.old_start[c + 1] - A.old_start[c] - lv + in[k] : 0;
                lmask |= (lv != 0 ? 1u : 0u) << k;
                imask |= (in[k] != 0 ? 1u : 0u) << k;
            }
        }
        uint32_t s = 0;
        // largest count of a grid cell that fits a tile (the overflow cell, the cloud's last, and the
        // dense cells are split across tiles)
        const int dense = dense_threshold(A.tile_cap);
        int m = 0;
#pragma unroll
        for (int k = 0; k < CELL_ITEMS; ++k) {
            s += (uint32_t)cnt[k];
            if (cb + k < cend - 1 && cnt[k] <= dense) m = max(m, cnt[k]);
        }
        m = (int)__reduce_max_sync(0xffffffffu, (unsigned)max(m, 0));
        if (lane == 0 && m > 0) atomicMax(&s_max, m);  // ordered by the scan's barriers
        uint32_t tot;
        const uint32_t ex = block_excl_scan_u32<CB>(s, wsum, tot);
        if (threadIdx.x < 32) {
            unsigned excl = 0;
            if (blk == 0) {
                if (lane == 0) lb_store(A.scan_desc, 0, lb_word(epoch, LB_INC, tot));
            } else if (MULTI && !A.init_mode && blk == head_blk) {
                // a cloud's first scan block in a physics step: its offset is the earlier clouds' new
                // totals, each its old total less the step's losses (atoms never change clouds), so
                // the chain restarts here and no block waits on the blocks of earlier clouds
                long long part = 0;
                for (int k2 = lane; k2 < hb.x; k2 += 32) part += A.cdyn[k2].n[A.parity] - A.cloud_lost[k2];
                excl = (unsigned)warp_sum_ll(part);
                if (lane == 0) lb_store(A.scan_desc, blk, lb_word(epoch, LB_INC, excl + tot));
            } else {
                if (lane == 0) lb_store(A.scan_desc, blk, lb_word(epoch, LB_AGG, tot));
                excl = lb_exclusive(A.scan_desc, blk, epoch, &A.ctl->err);
                if (lane == 0) lb_store(A.scan_desc, blk, lb_word(epoch, LB_INC, excl + tot));
            }
            if (lane == 0) s_excl = excl;
        }
        __syncthreads();
        int st = (int)(ex + s_excl);
        // one cloud in a physics step: the tiling of the coming step, built here with the current
        // nominal size (it starts at sorted position 0 and tile 0); kept by the top level when the
        // coming size turns out the same, else rebuilt where the atoms are placed
        const int Ts = spec ? A.ctl->tile_T[A.parity] : 0;
        int j = spec && Ts > 0 ? st / Ts + (st % Ts != 0) : 0;  // the first nominal start at or after st
#pragma unroll
        for (int v = 0; v < NV; ++v) {
            int o[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int k = 4 * v + u;
                o[u] = st;
                if ((imask >> k) & 1u) A.mover_base[cb + k] = st + cnt[k] - in[k];
                const int e = st + cnt[k];
                if (spec && Ts > 0) {
                    if (cb + k == cend - 1) {  // the overflow cell: its inner starts, below, by the block
                        if (j * Ts == st && st < e && j < A.max_tiles) {
                            A.tile_begin_next[j] = st;
                            A.tile_cloud_next[j] = 0;
                            A.tile_split_next[j] = 0;
                        }
                        s_ovf_st = st;
                        s_ovf_end = e;
                        j = e / Ts + (e % Ts != 0);
                    }
                    // nominal starts inside this cell snap to its end, unless the cell is dense
                    const bool spl = cnt[k] > dense && cb + k < cend - 1;
                    for (; j * Ts < e; ++j) {
                        const int pnom = j * Ts;
                        const int tbeg = (pnom == st || spl) ? pnom : e;
                        if (j < A.max_tiles) {
                            A.tile_begin_next[j] = tbeg;
                            A.tile_cloud_next[j] = 0;
                            A.tile_split_next[j] = tbeg != st && tbeg != e ? 1 : 0;
                        }
                    }
                }
                st = e;
            }
            if (whole) {
                *reinterpret_cast<int4*>(A.new_start + cb + 4 * v) = make_int4(o[0], o[1], o[2], o[3]);
                if ((lmask >> (4 * v)) & 15u) *reinterpret_cast<int4*>(A.Lc + cb + 4 * v) = make_int4(0, 0, 0, 0);
                if ((imask >> (4 * v)) & 15u) *reinterpret_cast<int4*>(A.Ic + cb + 4 * v) = make_int4(0, 0, 0, 0);
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int k = 4 * v + u;
                    if (cb + k < c1) A.new_start[cb + k] = o[u];
                    if ((lmask >> k) & 1u) A.Lc[cb + k] = 0;
                    if ((imask >> k) & 1u) A.Ic[cb + k] = 0;
                }
            }
        }
        // the overflow cell, which may hold many nominal starts: each begins a tile there (split)
        if (spec && Ts > 0 && c1 >= cend) {
            __syncthreads();
            const int ost = s_ovf_st, oend = s_ovf_end;
            for (int jj = ost / Ts + 1 + threadIdx.x; jj * Ts < oend; jj += CB) {
                if (jj < A.max_tiles) {
                    A.tile_begin_next[jj] = jj * Ts;
                    A.tile_cloud_next[jj] = 0;
                    A.tile_split_next[jj] = 1;
                }
            }
        }
    } else if (threadIdx.x == 0) {
        atomicOr(&A.ctl->err, EB_INCONSISTENT);  // more scan blocks than tickets: an earlier launch failed
    }
    if (threadIdx.x == 0) {
        if (s_max > 0) atomicMax(&A.ctl->max_cell, s_max);
        __threadfence();
        s_last = atomicAdd(&A.ctl->scan_done, 1) == A.nscan_blocks - 1;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if (threadIdx.x == 0) A.ctl->scan_done = 0;
    scan_top_block<R, CB>(A, epoch);
}

// Tile starts of the tiling the scan built after a full sort (no atoms are placed by
// permute_pass then): the same rule, per cell.
template <class R, int CB, int CELL_ITEMS>
__global__ void __launch_bounds__(CB) init_tiles(Args<R> A) {
    const int blk = blockIdx.x;
    const int4 hb = A.scan_blk[blk];
    const int cloud = hb.x, c0 = hb.y, cend = hb.z, c1 = hb.w;
    for (int k = 0; k < CELL_ITEMS; ++k) {
        const int c = c0 + threadIdx.x * CELL_ITEMS + k;
        if (c >= c1) break;
        const int st = A.new_start[c], e = A.new_start[c + 1];
        const bool dns = c != cend - 1 && e - st > dense_threshold(A.tile_cap);
        if (dns) list_dense(A, c, cloud);
        if (e > st) cell_tile_starts(A, cloud, st, e, c == cend - 1 || dns);
    }
}

// rank = number of incoming movers of the same cell with a smaller old position; unless scan_cells
// built the coming tiling, the mover placed at a grid cell's first position writes the cell's tile
// starts, every mover into a split cell (overflow or dense) checks its own position
template <class R>
__global__ void __launch_bounds__(256) mover_rank(Args<R> A) {
    const int m = min(A.ctl->movers[A.parity], A.mrec_cap);
    const bool tiles = A.ctl->tiles_built[1 - A.parity] == 0;  // the coming tiling is built here
    for (int i = blockIdx.x * 256 + threadIdx.x; i < m; i += gridDim.x * 256) {
        const int4 r = A.mrec[i];
        if (r.x < 0) continue;  // an unused slot of a warp's chunk
        A.Ic[r.x] = 0;  // the next step's incoming count starts at zero (every mover of the cell writes it)
        const int lo = A.mover_base[r.x];
        const int hi = A.new_start[r.x + 1];
        if (lo < 0 || hi > A.capacity || lo > hi) {
            atomicOr(&A.ctl->err, EB_INCONSISTENT);
            continue;
        }
        int rank = 0;
        for (int k = lo; k < hi; ++k) rank += (A.in_list[k] < r.y) ? 1 : 0;
        const int x = lo + rank;
        if (x < hi && r.y >= 0 && r.y < A.capacity) {
            A.src_out[x] = r.y;
            const int k = r.w & (MREC_OVF_CELL - 1);
            const int st = A.new_start[r.x];
            const bool ovf = (r.w & MREC_OVF_CELL) != 0;
            const bool dns = !ovf && hi - st > dense_threshold(A.tile_cap);
            if (dns && x == st) list_dense(A, r.x, k);
            if (tiles) {
                if (ovf || dns) {
                    split_tile_start(A, k, st, x);
                } else if (rank == 0) {
                    if (st == lo) cell_tile_starts(A, k, st, hi, false);
                }
            }
        } else {
            atomicOr(&A.ctl->err, EB_INCONSISTENT);
        }
    }
}

// diagnostics of the current (sorted) state without moving it: bucket totals for finalize<INIT>
template <class R, int BLOCK>
__global__ void __launch_bounds__(BLOCK) measure_tiles(Args<R> A) {
    typedef typename V4T<R>::type R4;
    __shared__ TilePartial red[BLOCK / 32];
    __shared__ CloudPhys<R> P;
    const int p = A.parity;
    const int ntiles = A.ctl->ntiles[p];
    for (int b = blockIdx.x; b < ntiles; b += gridDim.x) {
    const int tb = A.tile_begin[b], te = A.tile_begin[b + 1];
    load_cloud(P, A.clouds + A.tile_cloud[b]);
    __syncthreads();
    TilePartial acc;
    zero_partial(acc);
    for (int i = tb + threadIdx.x; i < te; i += BLOCK) {
        const int s = A.src_in[i];
        const R4 q = A.pos_in[s];
        const R4 v = A.vel_in[s];
        Field<R> f;
        trap_field(P, q.x, q.y, q.z, f);
        const R v2 = v.x * v.x + v.y * v.y + v.z * v.z;
        acc.n_alive += 1;
        acc.sum_v2 += fx_from(v2);
        acc.sum_B += fx_from((lane_to_u32(v.w) & 1u) ? -f.absB : f.absB);  // anti-trapped: -|B|
    }
    block_reduce_partial<BLOCK>(acc, red);
    if (threadIdx.x == 0) accum_tile(A.accum + A.tile_cloud[b] * ACC_BUCKETS + (b & (ACC_BUCKETS - 1)), acc);
    }
}

// ---------------------------------------------------------------------------------------------
// full sort (initialisation and set_state): arbitrary order -> stable by (cell, index).
// fs_cells finds every atom's global cell and counts the cells (the cell scan turns the counts
// into the sorted starts); the stable radix sort of the cell ids (dsmc_radix.cuh) gives, for
// every sorted position j, the source index order[j]; fs_gather copies the state there.
// ---------------------------------------------------------------------------------------------
template <class R> struct SortArgs {
    typedef typename V4T<R>::type R4;
    const R4* pos_src;
    const R4* vel_src;
    const R4* psi_src;
    R4* pos_dst;
    R4* vel_dst;
    R4* psi_dst;
    const int* cloud_atom_off;  // nclouds + 1, atoms of the source grouped by cloud
    int* cell;                  // global cell of each source atom
    const int* order;           // sorted position -> source index (after the radix sort)
    int n, nclouds;
};

template <class R>
__device__ __forceinline__ int find_cloud(const int* off, int nclouds, int i) {
    int lo = 0, hi = nclouds;  // off[lo] <= i < off[hi]
    while (hi - lo > 1) {
        const int mid = (lo + hi) >> 1;
        if (off[mid] <= i) lo = mid; else hi = mid;
    }
    return lo;
}

template <class R>
__global__ void __launch_bounds__(256) fs_cells(SortArgs<R> S, Args<R> A) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    const bool valid = i < S.n;
    int c = -1;
    if (valid) {
        const int k = find_cloud<R>(S.cloud_atom_off, S.nclouds, i);
        const CloudPhys<R>& P = A.clouds[k];
        const auto q = S.pos_src[i];
        c = cell_of(P, q.x, q.y, q.z, P.trap == TRAP_BOX);
        S.cell[i] = c;
    }
    // one atomic per cell and warp: input that is already nearly sorted (a state read back from
    // the engine) has runs of equal cells
    const unsigned vm = __ballot_sync(0xffffffffu, valid);
    if (valid) {
        const unsigned peers = __match_any_sync(vm, c);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&A.Ic[c], __popc(peers));
    }
}

template <class R>
__global__ void __launch_bounds__(256) fs_gather(SortArgs<R> S) {
    const int j = blockIdx.x * 256 + threadIdx.x;
    if (j >= S.n) return;
    const int i = S.order[j];
    S.pos_dst[j] = S.pos_src[i];
    S.vel_dst[j] = S.vel_src[i];
    S.psi_dst[j] = S.psi_src[i];
}

// generic exclusive scan of n ints (3 kernels, no inter-block waiting)
__global__ void __launch_bounds__(SCAN_BLOCK) gscan_reduce(const int* in, int n, int* bsum) {
    __shared__ uint32_t wsum[32];
    const int base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_ITEMS;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k)
        if (base + k < n) s += (uint32_t)in[base + k];
    uint32_t tot;
    block_excl_scan_u32<SCAN_BLOCK>(s, wsum, tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = (int)tot;
}
__global__ void __launch_bounds__(1024) gscan_top(int* bsum, int nb, int* total) {
    __shared__ uint32_t wsum[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += 1024) {
        const int i = base + threadIdx.x;
        const uint32_t v = i < nb ? (uint32_t)bsum[i] : 0u;
        uint32_t tot;
        const uint32_t ex = block_excl_scan_u32<1024>(v, wsum, tot);
        if (i < nb) bsum[i] = (int)ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += (int)tot;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total) *total = carry;
}
__global__ void __launch_bounds__(SCAN_BLOCK) gscan_down(const int* in, int n, const int* boff, int* out) {
    __shared__ uint32_t wsum[32];
    const int base = blockIdx.x * SCAN_CHUNK + threadIdx.x * SCAN_ITEMS;
    int v[SCAN_ITEMS];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += (uint32_t)v[k];
    }
    uint32_t tot;
    uint32_t ex = block_excl_scan_u32<SCAN_BLOCK>(s, wsum, tot) + (uint32_t)boff[blockIdx.x];
#pragma unroll
    for (int k = 0; k < SCAN_ITEMS; ++k) {
        if (base + k < n) out[base + k] = (int)ex;
        ex += (uint32_t)v[k];
    }
}

// ---------------------------------------------------------------------------------------------
// initial cloud and small fills
// ---------------------------------------------------------------------------------------------
template <class R>
__global__ void __launch_bounds__(256) init_atoms(Args<R> A, const int* cloud_atom_off, int n,
                                                  const int* init_mode, typename V4T<R>::type* pos,
                                                  typename V4T<R>::type* vel, typename V4T<R>::type* psi,
                                                  unsigned long long seed) {
    typedef typename V4T<R>::type R4;
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i >= n) return;
    const int k = find_cloud<R>(cloud_atom_off, A.nclouds, i);
    const CloudPhys<R>& P = A.clouds[k];
    const uint32_t local = (uint32_t)(i - cloud_atom_off[k]);
    Atom<R> a;
    const bool ok = init_atom(P, init_mode[k], local, (uint64_t)seed, a);
    if (!ok) atomicOr(&A.ctl->err, EB_INIT_REJECT);
    R4 q, v, s;
    q.x = a.x; q.y = a.y; q.z = a.z; q.w = lane_from_u32(local, R(0));
    v.x = a.vx; v.y = a.vy; v.z = a.vz; v.w = lane_from_u32(a.flags, R(0));
    s.x = a.ur; s.y = a.ui; s.z = a.dr; s.w = a.di;
    pos[i] = q;
    vel[i] = v;
    psi[i] = s;
}

// sorted copy of the current state (for get_state): out[j] = state[src[j]]
template <class R>
__global__ void __launch_bounds__(256) materialize(Args<R> A, int n, typename V4T<R>::type* pos,
                                                   typename V4T<R>::type* vel, typename V4T<R>::type* psi) {
    const int j = blockIdx.x * 256 + threadIdx.x;
    if (j >= n) return;
    const int s = A.src_in[j];
    pos[j] = A.pos_in[s];
    vel[j] = A.vel_in[s];
    psi[j] = A.psi_in[s];
}

__global__ void fill_identity(int* a, int n) {
    const int i = blockIdx.x * 256 + threadIdx.x;
    if (i < n) a[i] = i;
}

template <class R>
__global__ void fill_sigvrmax(R* sv, const int* cell_cloud_base, const R* init_val, int nclouds, int total) {
    const int c = blockIdx.x * 256 + threadIdx.x;
    if (c >= total) return;
    int k = 0;
    while (k + 1 < nclouds && cell_cloud_base[k + 1] <= c) ++k;
    sv[c] = init_val[k];
}

}  // namespace dsmc

#endif  // DSMC_KERNELS_CUH

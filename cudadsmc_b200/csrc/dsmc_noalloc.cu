// dsmc_noalloc.cu -- cell sort of caller-owned device positions that allocates no memory.
//
// Callers that own all device memory through their own allocator (for example a PyTorch
// process whose caching allocator already holds the GPU's memory) cannot rely on cudaMalloc:
// it can fail for lack of free memory the pool is holding, and cudaMalloc / cudaFree
// synchronise the device, stalling every other stream of the application.  For them this
// entry point sorts one cloud's atoms by cell using only a fixed scratch region compiled into
// the library (g_noalloc_scratch below, about 5.3 MB, held by every GPU that loads the library
// until the process exits).  The caller passes device pointers for the input positions and for
// both outputs; nothing is allocated or freed.
//
// The order it produces is the engine's full-sort order: stable by (cell, input index), where
// the cell id and the overflow cell are those of the engine (grid cells z*nx*ny + y*nx + x, then
// the overflow cell for atoms outside the grid).  It is the engine's stable radix sort of the
// cell ids (dsmc_radix.cuh), so its time grows with the atoms, whatever the cells hold.
#include <cuda_runtime.h>

#include <mutex>
#include <string>
#include <type_traits>

#include "dsmc.h"
#include "dsmc_physics.h"
#include "dsmc_radix.cuh"
#include "dsmc_setup.h"

namespace {

using namespace dsmc;

constexpr int kMaxAtoms = 1 << 18;          // atoms per call
constexpr int kMaxCells = (1 << 18) + 1;    // grid cells + overflow cell per call (64^3 + 1)
constexpr int kBlock = 256;
constexpr int kItems = 8;
constexpr int kChunk = kBlock * kItems;     // elements per scan block
constexpr int kMaxTable = RADIX_DIGITS * ((kMaxAtoms + RADIX_CHUNK - 1) / RADIX_CHUNK);  // digit counts of a pass
constexpr int kMaxScanLen = kMaxCells > kMaxTable ? kMaxCells : kMaxTable;
constexpr int kMaxScanBlocks = (kMaxScanLen + kChunk - 1) / kChunk + 1;

// layout of the scratch (ints): per-cell counters, the radix keys and values (two ping-pong
// pairs; the first keys are the atoms' cells), the digit count table, then scan block sums
constexpr int kOffCounts = 0;
constexpr int kOffKeyA = kOffCounts + kMaxCells + 1;
constexpr int kOffKeyB = kOffKeyA + kMaxAtoms;
constexpr int kOffValA = kOffKeyB + kMaxAtoms;
constexpr int kOffValB = kOffValA + kMaxAtoms;
constexpr int kOffTable = kOffValB + kMaxAtoms;
constexpr int kOffBlocks = kOffTable + kMaxTable;
constexpr int kScratchInts = kOffBlocks + kMaxScanBlocks + 1;

static __device__ __align__(256) int g_noalloc_scratch[kScratchInts];

// Device address of the scratch, looked up once per device with that device current, and again
// when the device's current context is no longer the one of the lookup (after a
// cudaDeviceReset the module is loaded anew and the array may sit elsewhere).
constexpr int kMaxDevices = 64;
struct ScratchAddr {
    int* addr;
    void* ctx;
};
ScratchAddr g_scratch_addr[kMaxDevices] = {};
std::mutex g_scratch_mutex;

// the driver's cuCtxGetCurrent through the runtime (no link against the driver library)
typedef int (*CtxGetCurrentFn)(void**);
CtxGetCurrentFn ctx_get_current() {
    static CtxGetCurrentFn fn = nullptr;
    static bool looked = false;
    if (!looked) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<CtxGetCurrentFn>(f);
        looked = true;
    }
    return fn;
}

cudaError_t scratch_for_current_device(int** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_scratch_mutex);
    // the current context (null until the runtime has made the device's context current, which
    // the symbol lookup does)
    CtxGetCurrentFn get = ctx_get_current();
    void* ctx = nullptr;
    if (get && get(&ctx) != 0) ctx = nullptr;
    ScratchAddr& s = g_scratch_addr[dev];
    if (!s.addr || !ctx || s.ctx != ctx) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e != cudaSuccess) return e;
        if (get && get(&ctx) != 0) ctx = nullptr;
        s.addr = static_cast<int*>(p);
        s.ctx = ctx;
    }
    *out = s.addr;
    return cudaSuccess;
}

template <int BLOCK>
__device__ __forceinline__ uint32_t excl_scan(uint32_t v, uint32_t* wsum, uint32_t& total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = BLOCK / 32;
    uint32_t x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const uint32_t y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) wsum[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t w = lane < NW ? wsum[lane] : 0u;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t y = __shfl_up_sync(0xffffffffu, w, o);
            if (lane >= o) w += y;
        }
        if (lane < NW) wsum[lane] = w;
    }
    __syncthreads();
    const uint32_t off = warp ? wsum[warp - 1] : 0u;
    total = wsum[NW - 1];
    __syncthreads();
    return off + x - v;
}

__global__ void k_zero(int* a, int n) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    if (i < n) a[i] = 0;
}

template <class R4, class R>
__global__ void k_cells(const R4* pos, int n, CloudPhys<R> P, int* scratch) {
    const int i = blockIdx.x * kBlock + threadIdx.x;
    const bool valid = i < n;
    int c = -1;
    if (valid) {
        const R4 q = pos[i];
        c = cell_of(P, q.x, q.y, q.z, P.trap == TRAP_BOX);  // ids start at 0 (cell_base 0)
        scratch[kOffKeyA + i] = c;
    }
    // one atomic per cell and warp (runs of equal cells in nearly sorted input)
    const unsigned vm = __ballot_sync(0xffffffffu, valid);
    if (valid) {
        const unsigned peers = __match_any_sync(vm, c);
        if ((threadIdx.x & 31) == __ffs(peers) - 1) atomicAdd(&scratch[kOffCounts + c], __popc(peers));
    }
}

// exclusive scan of in[0..n) into out[0..n) (3 kernels, block sums in the scratch)
__global__ void k_scan_reduce(const int* in, int n, int* bsum) {
    __shared__ uint32_t wsum[32];
    const int base = blockIdx.x * kChunk + threadIdx.x * kItems;
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k)
        if (base + k < n) s += (uint32_t)in[base + k];
    uint32_t tot;
    excl_scan<kBlock>(s, wsum, tot);
    if (threadIdx.x == 0) bsum[blockIdx.x] = (int)tot;
}
__global__ void k_scan_top(int* bsum, int nb, int* total_out) {
    __shared__ uint32_t wsum[32];
    __shared__ int carry;
    if (threadIdx.x == 0) carry = 0;
    __syncthreads();
    for (int base = 0; base < nb; base += 1024) {
        const int i = base + threadIdx.x;
        const uint32_t v = i < nb ? (uint32_t)bsum[i] : 0u;
        uint32_t tot;
        const uint32_t ex = excl_scan<1024>(v, wsum, tot);
        if (i < nb) bsum[i] = (int)ex + carry;
        __syncthreads();
        if (threadIdx.x == 0) carry += (int)tot;
        __syncthreads();
    }
    if (threadIdx.x == 0 && total_out) *total_out = carry;
}
__global__ void k_scan_down(const int* in, int n, const int* boff, int* out) {
    __shared__ uint32_t wsum[32];
    const int base = blockIdx.x * kChunk + threadIdx.x * kItems;
    int v[kItems];
    uint32_t s = 0;
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        v[k] = (base + k < n) ? in[base + k] : 0;
        s += (uint32_t)v[k];
    }
    uint32_t tot;
    uint32_t ex = excl_scan<kBlock>(s, wsum, tot) + (uint32_t)boff[blockIdx.x];
#pragma unroll
    for (int k = 0; k < kItems; ++k) {
        if (base + k < n) out[base + k] = (int)ex;
        ex += (uint32_t)v[k];
    }
}

void scan(const int* in, int n, int* out, int* bsum, int* total, cudaStream_t s) {
    const int nb = (n + kChunk - 1) / kChunk;
    k_scan_reduce<<<nb, kBlock, 0, s>>>(in, n, bsum);
    k_scan_top<<<1, 1024, 0, s>>>(bsum, nb, total);
    k_scan_down<<<nb, kBlock, 0, s>>>(in, n, bsum, out);
}

template <class R>
dsmc_status sort_cells(const dsmc_params& rp, const dsmc_cloud_params& cp, const void* pos, int n, int32_t* order,
                int32_t* cell_start, cudaStream_t s, int* scratch) {
    typedef typename std::conditional<sizeof(R) == 4, float4, double4>::type R4;
    CloudPhys<R> P;
    make_cloud_phys<R>(rp, cp, 0, 0, P);
    const int ncells = P.ovf_cell + 1;  // grid cells + overflow cell
    const int ab = (n + kBlock - 1) / kBlock;
    // the scratch keeps the previous call's contents: the counters must start at zero
    k_zero<<<(ncells + kBlock - 1) / kBlock, kBlock, 0, s>>>(scratch + kOffCounts, ncells);
    if (n > 0) k_cells<R4, R><<<ab, kBlock, 0, s>>>(static_cast<const R4*>(pos), n, P, scratch);
    // cell starts (the caller's output) and the total in cell_start[ncells]
    scan(scratch + kOffCounts, ncells, cell_start, scratch + kOffBlocks, cell_start + ncells, s);
    if (n > 0) {
        // stable by (cell, input index): LSD passes over the digits of the cell ids, the last one
        // writing the caller's order
        int* const key[2] = {scratch + kOffKeyA, scratch + kOffKeyB};
        int* const val[2] = {scratch + kOffValA, scratch + kOffValB};
        int* const table = scratch + kOffTable;
        const int nch = radix_chunks(n), passes = radix_passes(ncells);
        const int tsize = (int)radix_table(n);
        for (int q = 0; q < passes; ++q) {
            const bool last = q + 1 == passes;
            radix_hist<<<nch, RADIX_BLOCK, 0, s>>>(key[q & 1], n, RADIX_BITS * q, table, nch);
            scan(table, tsize, table, scratch + kOffBlocks, nullptr, s);
            radix_scatter<<<nch, RADIX_BLOCK, 0, s>>>(key[q & 1], q == 0 ? nullptr : val[q & 1], n, RADIX_BITS * q,
                                                      table, nch, last ? nullptr : key[(q + 1) & 1],
                                                      last ? order : val[(q + 1) & 1]);
        }
    }
    const cudaError_t e = cudaGetLastError();
    return e == cudaSuccess ? DSMC_OK : DSMC_ERR_CUDA;
}

}  // namespace

DSMC_API dsmc_status dsmc_sort_cells_noalloc(const dsmc_params* run, const dsmc_cloud_params* cloud,
                                             const void* pos_dev, int64_t n, int32_t* order_dev,
                                             int32_t* cell_start_dev, void* cuda_stream) {
    if (!run || !cloud || n < 0 || (n > 0 && (!pos_dev || !order_dev)) || !cell_start_dev) return DSMC_ERR_INVALID;
    if (!validate_cloud(*run, *cloud, 0).empty()) return DSMC_ERR_INVALID;
    if (n > kMaxAtoms) return DSMC_ERR_CAPACITY;
    if (cloud_cells(*cloud) > kMaxCells) return DSMC_ERR_CAPACITY;
    if (run->precision != DSMC_FP32 && run->precision != DSMC_FP64) return DSMC_ERR_INVALID;
    // the positions are read as 16-byte (float4) or 32-byte (double4) vectors
    const uintptr_t align = run->precision == DSMC_FP32 ? 16u : 32u;
    if (n > 0 && ((uintptr_t)pos_dev % align) != 0) return DSMC_ERR_INVALID;
    // an error left pending on this thread by earlier work is the caller's: report it untouched
    if (cudaPeekAtLastError() != cudaSuccess) return DSMC_ERR_STATE;
    int* scratch = nullptr;
    if (scratch_for_current_device(&scratch) != cudaSuccess) return DSMC_ERR_CUDA;
    cudaStream_t s = static_cast<cudaStream_t>(cuda_stream);
    if (run->precision == DSMC_FP32)
        return sort_cells<float>(*run, *cloud, pos_dev, (int)n, order_dev, cell_start_dev, s, scratch);
    return sort_cells<double>(*run, *cloud, pos_dev, (int)n, order_dev, cell_start_dev, s, scratch);
}

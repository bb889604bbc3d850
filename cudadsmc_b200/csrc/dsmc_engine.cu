// dsmc_engine.cu -- host side of the B200 DSMC engine: handle, device memory, launch
// sequence of one timestep (captured into CUDA graphs), full sort, diagnostics and the C ABI
// declared in include/dsmc.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dsmc.h"
#include "dsmc_adjoint.cuh"
#include "dsmc_kernels.cuh"
#include "dsmc_setup.h"

using namespace dsmc;

namespace {

struct Fail {
    dsmc_status st;
    std::string msg;
};

#define CU(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess)                                                                     \
            throw Fail{e_ == cudaErrorMemoryAllocation ? DSMC_ERR_ALLOC : DSMC_ERR_CUDA,           \
                       std::string(#call) + ": " + cudaGetErrorString(e_)};                        \
    } while (0)

template <class T> struct DevBuf {
    T* p = nullptr;
    size_t n = 0;
    void alloc(size_t count) {
        free();
        n = count;
        if (count) CU(cudaMalloc((void**)&p, count * sizeof(T)));
    }
    void free() {
        if (p) cudaFree(p);
        p = nullptr;
        n = 0;
    }
    ~DevBuf() { free(); }
};

constexpr int kMinTile = MIN_TILE;  // smallest tile the autotuner tries (sizes the tile tables)

// launch shape of the FP32 step_pass: threads per tile, atoms staged per tile (42 B of shared
// memory each: position and velocity, storage index, cell, head), blocks per SM requested from
// the compiler
#ifndef DSMC_FP32_BLOCK
#define DSMC_FP32_BLOCK 256
#endif
#ifndef DSMC_FP32_CAP
#define DSMC_FP32_CAP 1280
#endif
#ifndef DSMC_FP32_MINB
#define DSMC_FP32_MINB 4
#endif

// the kernels of one step, in launch order
const char* kKernelNames[] = {"dense_collide", "step_pass", "scan_cells", "permute_pass", "mover_rank"};
constexpr int kNumStepKernels = 5;

}  // namespace

struct dsmc_handle {
    std::string last_error;
    virtual ~dsmc_handle() {}
    virtual void init(uint64_t seed) = 0;
    virtual void step(int n) = 0;
    virtual void sync() = 0;
    virtual void diag(int cloud, dsmc_diag* out) = 0;
    virtual void diag_reserve(int nslots) = 0;
    virtual void diag_enqueue(int slot) = 0;
    virtual void diag_collect(int slot, int cloud, dsmc_diag* out) = 0;
    virtual int64_t diag_copy_bytes() const = 0;
    virtual void get_state(dsmc_state_buffers* out) = 0;
    virtual void set_state(const dsmc_state_buffers* in) = 0;
    virtual void get_cell_starts(int32_t* start, int64_t cap, int64_t* total) = 0;
    virtual void get_sigvrmax(void* out, int64_t cap) = 0;
    virtual void set_sigvrmax(const void* in, int64_t n) = 0;
    virtual void set_stream(cudaStream_t s) = 0;
    virtual void set_profiling(bool on) = 0;
    virtual void kernel_times(const char** names, double* ms, int64_t* launches, int cap, int* count) = 0;
    virtual int check_wait_timeout() = 0;
    virtual void autotune(int steps_per_candidate, int32_t* chosen, double* ms_per_step) = 0;
    virtual void autotune_table(int32_t* T, int32_t* B, double* ms, int cap, int32_t* count, int32_t* chosen_b) = 0;
    virtual void adjoint_run(const dsmc_adj_params* p, dsmc_grad* g) = 0;
    virtual void adjoint_loss(const double* theta, double* parts, double* grad_e, double* grad_n) = 0;
    virtual void adjoint_export_spinors(double* psi0, int64_t atoms_cap) = 0;
    virtual void set_recording(int flags) = 0;
    virtual void get_evaporated(int cloud, double* pos3, double* vel3, int32_t* step, int32_t* fate, int64_t cap) = 0;
    virtual void get_cell_collisions(int32_t* counts, int64_t cap, int64_t* total) = 0;
    virtual void adjoint_export(double* x0, double* v0, int64_t atoms_cap, int32_t* off, int64_t off_cap, int32_t* ij,
                                double* nv, int64_t log_cap, int64_t* n_atoms, int64_t* n_log, int32_t* steps) = 0;
};

namespace {

// BLOCK threads per step_pass tile, CAP atoms staged per tile, MINB blocks per SM requested
template <class R, int BLOCK, int CAP, int MINB> struct Engine final : dsmc_handle {
    typedef typename V4T<R>::type R4;
    // configuration
    dsmc_params run{};
    std::vector<dsmc_cloud_params> cp;
    std::vector<CloudPhys<R>> phys;
    int nclouds = 0;
    int total_cells = 0;
    int capacity = 0;
    int max_tiles = 0;
    int tile_nominal = 0;
    int nscan_blocks = 0;
    int cell_items = 16;  // cells per thread of a scan_cells block (cell_items_for)
    std::vector<int> cloud_atoms_init;  // initial atoms per cloud
    std::vector<int> cloud_cell_base;
    // device memory
    DevBuf<R4> pos[2], vel[2], psi[2];
    DevBuf<int> start[2], tile_begin[2], tile_cloud[2], tile_split[2];
    DevBuf<int> src[2];
    DevBuf<int> Lc, Ic, mover_base, in_list, tile_ovf, tile_ovf_carry, ovf_list, tile_cell;
    DevBuf<int2> dense_list;
    DevBuf<int> cloud_lost;  // per cloud: atoms removed by the current step (read and cleared by its scan)
    int dense_cap = 0;  // dense cells a step can hold: each has more than dense_threshold(CAP) atoms
    DevBuf<int4> mrec;
    DevBuf<int2> keys;
    DevBuf<R> sigvrmax;
    DevBuf<CloudAccum> accum;
    DevBuf<CloudPhys<R>> d_phys;
    DevBuf<CloudDyn> cdyn;
    DevBuf<CloudDiagDev> cdiag;
    DevBuf<Ctl> ctl;
    DevBuf<unsigned long long> scan_desc;  // LB_STRIDE words per scan block
    DevBuf<int4> scan_blk;
    DevBuf<int> cloud_first_blk, d_cell_base, sort_off, init_modes;
    DevBuf<R> init_sv;
    // runtime
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int parity = 0;
    bool initialised = false;
    int64_t steps_taken = 0;
    Args<R> args[2];
    cudaGraphExec_t graph2 = nullptr;  // two steps: parity 0 then 1
    cudaGraphExec_t graph1[2] = {nullptr, nullptr};  // one step of each parity (odd step counts)
    bool use_graphs = true;
    bool profiling = false;
    double prof_ms[kNumStepKernels] = {0};
    int64_t prof_n[kNumStepKernels] = {0};
    cudaEvent_t ev[kNumStepKernels + 1] = {};  // also reused by the autotuner and the adjoint (>= 4)
    size_t smem_tile = 0;
    // resident blocks of the tile kernels on the whole device (their grid-stride loops cover
    // any tile count, so a launch never needs more blocks than fit at once)
    int resident_step = 0, resident_permute = 0, resident_measure = 0;
    int num_sms = 0, step_occ = 0;  // SMs, and step-kernel blocks that fit on one SM
    int step_bps = 0;               // step-kernel blocks per SM in use (<= step_occ)

    Engine(const dsmc_params& r, const dsmc_cloud_params* clouds, int n) {
        run = r;
        nclouds = n;
        cp.assign(clouds, clouds + n);
        use_graphs = r.use_graphs != 0;
        // preferred nominal tile: three passes of the block, less a part of a cell for the snap
        // to cell boundaries (each step's scan lowers it where a cell that is not split across
        // tiles is fuller than CAP - T + 1)
        tile_nominal = r.tile_atoms > 0 ? r.tile_atoms : CAP - BLOCK - 16;
        // a tile of nominal size T fits every cell of up to CAP - T + 1 atoms beside it
        if (tile_nominal > CAP - 128) throw Fail{DSMC_ERR_INVALID, "tile_atoms must be <= " + std::to_string(CAP - 128)};
        if (tile_nominal < kMinTile) throw Fail{DSMC_ERR_INVALID, "tile_atoms must be >= " + std::to_string(kMinTile)};
        build_phys();
        allocate();
        CU(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
        own_stream = true;
        for (int i = 0; i <= kNumStepKernels; ++i) CU(cudaEventCreate(&ev[i]));
        int dev = 0, nsm = 0, occ = 0;
        CU(cudaGetDevice(&dev));
        CU(cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev));
        smem_tile = (size_t)CAP * (2 * sizeof(R4) + 2 * sizeof(int) + sizeof(uint16_t));
        CU(cudaFuncSetAttribute(dense_collide<R>, cudaFuncAttributeMaxDynamicSharedMemorySize, DENSE_SMEM_BYTES));
        CU(cudaFuncSetAttribute(step_pass<R, BLOCK, CAP, MINB, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem_tile));
        CU(cudaFuncSetAttribute(step_pass<R, BLOCK, CAP, MINB, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)smem_tile));
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, step_pass<R, BLOCK, CAP, MINB, false>, BLOCK, smem_tile));
        num_sms = nsm;
        step_occ = std::max(occ, 1);
        step_bps = (r.step_blocks_per_sm > 0 && r.step_blocks_per_sm < step_occ) ? r.step_blocks_per_sm : step_occ;
        resident_step = nsm * step_bps;
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, permute_pass<R>, 256, 0));
        resident_permute = nsm * std::max(occ, 1);
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, measure_tiles<R, 256>, 256, 0));
        resident_measure = nsm * std::max(occ, 1);
        build_args();
    }

    // blocks for a tile kernel: no more than the tiles of a tiling of the current nominal size
    // (a cloud of n atoms has at most n / T + 1 tiles) nor than fit on the device at once
    int tile_grid(int resident) const {
        // the smallest nominal size the scan may pick: one block pass when it adapts to the run
        const int tmin = args[0].tile_fill > 0 ? std::min(tile_nominal, BLOCK - 16) : tile_nominal;
        const int bound = capacity / tmin + nclouds + 2;
        return std::max(1, std::min(bound, resident));
    }

    // mover-list entries beyond the capacity: each resident step_pass warp (at most 64 per SM) may
    // leave up to MV_CHUNK - 1 slots of its last chunk unused
    int num_sms_dev = 0;
    int mover_slack() const { return num_sms_dev * 64 * MV_CHUNK; }
    int mover_list_size() const { return (int)std::min<int64_t>((int64_t)capacity + mover_slack(), INT32_MAX); }

    // blocks of the step kernel: no more than the tiles of the smallest tiling the scan may build
    // nor than the chosen number that run at once
    int step_grid() const { return tile_grid(resident_step); }

    ~Engine() override {
        drop_graphs();
        free_diag_slots();
        for (int i = 0; i <= kNumStepKernels; ++i)
            if (ev[i]) cudaEventDestroy(ev[i]);
        if (own_stream && stream) cudaStreamDestroy(stream);
    }

    // ------------------------------------------------------------------ parameters
    void build_phys() {
        phys.resize(nclouds);
        cloud_cell_base.resize(nclouds + 1);
        cloud_atoms_init.resize(nclouds);
        int64_t cells = 0, cap = 0;
        for (int k = 0; k < nclouds; ++k) {
            const dsmc_cloud_params& c = cp[k];
            const std::string bad = validate_cloud(run, c, k);
            if (!bad.empty()) throw Fail{DSMC_ERR_INVALID, bad};
            if (cells + cloud_cells(c) >= ((int64_t)1 << 31)) throw Fail{DSMC_ERR_INVALID, "more than 2^31 cells"};
            make_cloud_phys<R>(run, c, k, (int)cells, phys[k]);
            cloud_cell_base[k] = (int)cells;
            cells += cloud_cells(c);
            const int64_t ck = c.capacity > 0 ? c.capacity : c.n_atoms;
            phys[k].id_base = (int32_t)std::min<int64_t>(cap, INT32_MAX);
            phys[k].id_cap = (int32_t)std::min<int64_t>(ck, INT32_MAX);
            cap += ck;
            cloud_atoms_init[k] = (int)c.n_atoms;
        }
        cloud_cell_base[nclouds] = (int)cells;
        if (cap >= ((int64_t)1 << 31)) throw Fail{DSMC_ERR_INVALID, "more than 2^31 atoms"};
        total_cells = (int)cells;
        capacity = (int)std::max<int64_t>(cap, 1);
        max_tiles = capacity / std::min(tile_nominal, kMinTile) + nclouds + 2;
    }

    void allocate() {
        {
            int dev = 0;
            CU(cudaGetDevice(&dev));
            CU(cudaDeviceGetAttribute(&num_sms_dev, cudaDevAttrMultiProcessorCount, dev));
        }
        for (int i = 0; i < 2; ++i) {
            pos[i].alloc(capacity); vel[i].alloc(capacity); psi[i].alloc(capacity);
            src[i].alloc(capacity);
            start[i].alloc(total_cells + 1);
            tile_begin[i].alloc(max_tiles + 1);
            tile_cloud[i].alloc(max_tiles);
            tile_split[i].alloc(max_tiles);
            CU(cudaMemset(start[i].p, 0, (total_cells + 1) * sizeof(int)));
            CU(cudaMemset(tile_begin[i].p, 0, (max_tiles + 1) * sizeof(int)));
            CU(cudaMemset(tile_cloud[i].p, 0, max_tiles * sizeof(int)));
            CU(cudaMemset(tile_split[i].p, 0, max_tiles * sizeof(int)));
        }
        Lc.alloc(total_cells); Ic.alloc(total_cells); mover_base.alloc(total_cells);
        CU(cudaMemset(Lc.p, 0, total_cells * sizeof(int)));
        CU(cudaMemset(Ic.p, 0, total_cells * sizeof(int)));
        in_list.alloc(capacity);
        mrec.alloc(mover_list_size());
        keys.alloc(std::max(capacity, 2048));  // >= 4096 ints: the full sort's count table
        tile_ovf.alloc(max_tiles); tile_ovf_carry.alloc(max_tiles); ovf_list.alloc(max_tiles);
        tile_cell.alloc(max_tiles);
        dense_cap = capacity / (dense_threshold(CAP) + 1) + 1;
        dense_list.alloc(dense_cap);
        cloud_lost.alloc(nclouds);
        CU(cudaMemset(cloud_lost.p, 0, nclouds * sizeof(int)));
        sigvrmax.alloc(total_cells);
        accum.alloc((size_t)nclouds * ACC_BUCKETS);
        CU(cudaMemset(accum.p, 0, (size_t)nclouds * ACC_BUCKETS * sizeof(CloudAccum)));
        d_phys.alloc(nclouds);
        CU(cudaMemcpy(d_phys.p, phys.data(), nclouds * sizeof(CloudPhys<R>), cudaMemcpyHostToDevice));
        cdyn.alloc(nclouds); cdiag.alloc(nclouds); ctl.alloc(1);
        CU(cudaMemset(cdyn.p, 0, nclouds * sizeof(CloudDyn)));
        CU(cudaMemset(cdiag.p, 0, nclouds * sizeof(CloudDiagDev)));
        CU(cudaMemset(ctl.p, 0, sizeof(Ctl)));
        // scan blocks: each covers up to CELL_BLOCK * cell_items cells of a single cloud
        cell_items = cell_items_for(total_cells);
        const int chunk = CELL_BLOCK * cell_items;
        std::vector<int4> hb;
        std::vector<int> first(nclouds + 1);
        // a cloud whose cells start off a 4-cell boundary gets a first block of the 1-3 cells up to
        // it, so that its full blocks start on 16-byte boundaries (vector loads and stores)
        for (int k = 0; k < nclouds; ++k) {
            first[k] = (int)hb.size();
            const int c_beg = cloud_cell_base[k], c_end = cloud_cell_base[k + 1];
            int c = c_beg;
            const int c_al = std::min((c_beg + 3) & ~3, c_end);
            if (c_al > c) {
                hb.push_back(make_int4(k, c, c_end, c_al));
                c = c_al;
            }
            for (; c < c_end; c += chunk) hb.push_back(make_int4(k, c, c_end, std::min(c + chunk, c_end)));
        }
        first[nclouds] = (int)hb.size();
        nscan_blocks = (int)hb.size();
        scan_blk.alloc(nscan_blocks); cloud_first_blk.alloc(nclouds + 1);
        scan_desc.alloc((size_t)nscan_blocks * LB_STRIDE);
        CU(cudaMemset(scan_desc.p, 0, (size_t)nscan_blocks * LB_STRIDE * sizeof(unsigned long long)));
        d_cell_base.alloc(nclouds + 1);
        sort_off.alloc(nclouds + 1);
        init_modes.alloc(nclouds);
        init_sv.alloc(nclouds);
        CU(cudaMemcpy(d_cell_base.p, cloud_cell_base.data(), (nclouds + 1) * sizeof(int), cudaMemcpyHostToDevice));
        CU(cudaMemcpy(scan_blk.p, hb.data(), nscan_blocks * sizeof(int4), cudaMemcpyHostToDevice));
        CU(cudaMemcpy(cloud_first_blk.p, first.data(), (nclouds + 1) * sizeof(int), cudaMemcpyHostToDevice));
    }

    void build_args() {
        for (int p = 0; p < 2; ++p) {
            Args<R>& A = args[p];
            memset(&A, 0, sizeof(A));
            const int q = 1 - p;
            A.pos_in = pos[p].p; A.vel_in = vel[p].p; A.psi_in = psi[p].p;
            A.pos_out = pos[q].p; A.vel_out = vel[q].p; A.psi_out = psi[q].p;
            A.src_in = src[p].p; A.src_out = src[q].p; A.keys = keys.p;
            A.old_start = start[p].p; A.new_start = start[q].p;
            A.Lc = Lc.p; A.Ic = Ic.p; A.mover_base = mover_base.p;
            A.sigvrmax = sigvrmax.p;
            A.mrec = mrec.p; A.mrec_cap = mover_list_size(); A.in_list = in_list.p;
            A.tile_begin = tile_begin[p].p; A.tile_cloud = tile_cloud[p].p; A.tile_split = tile_split[p].p;
            A.tile_begin_next = tile_begin[q].p; A.tile_cloud_next = tile_cloud[q].p;
            A.tile_split_next = tile_split[q].p;
            A.tile_ovf = tile_ovf.p; A.tile_ovf_carry = tile_ovf_carry.p; A.ovf_list = ovf_list.p;
            A.tile_cell = tile_cell.p; A.dense_list = dense_list.p; A.dense_cap = dense_cap;
            A.cloud_lost = cloud_lost.p;
            A.accum = accum.p;
            A.clouds = d_phys.p; A.cdyn = cdyn.p; A.cdiag = cdiag.p; A.ctl = ctl.p;
            A.one = phys[0];
            A.scan_desc = scan_desc.p; A.cloud_cell_base = d_cell_base.p;
            A.scan_blk = scan_blk.p;
            A.cloud_first_blk = cloud_first_blk.p;
            A.nclouds = nclouds; A.total_cells = total_cells; A.nscan_blocks = nscan_blocks;
            A.max_tiles = max_tiles; A.tile_nominal = tile_nominal; A.tile_cap = CAP;
            A.tile_pass = BLOCK;
            A.tile_fill = run.tile_atoms > 0 ? 0 : resident_step;  // an explicit size is kept as given
            A.collide_every = run.collide_every; A.parity = p; A.init_mode = 0;
            A.seed = run.seed;
            A.capacity = capacity;
        }
    }

    // ------------------------------------------------------------------ launches
    void launch_step_kernel(int which, const Args<R>& A) {
        switch (which) {
        case 0: dense_collide<R><<<DENSE_GRID, DENSE_BLOCK, DENSE_SMEM_BYTES, stream>>>(A); break;
        case 1:
            if (nclouds == 1)
                step_pass<R, BLOCK, CAP, MINB, true><<<step_grid(), BLOCK, smem_tile, stream>>>(A);
            else
                step_pass<R, BLOCK, CAP, MINB, false><<<step_grid(), BLOCK, smem_tile, stream>>>(A);
            break;
        case 2: launch_scan(A, scan_extra_blocks(nclouds, CELL_BLOCK)); break;
        case 3: permute_pass<R><<<resident_permute, 256, 0, stream>>>(A); break;
        case 4: mover_rank<R><<<MOVER_GRID, 256, 0, stream>>>(A); break;
        }
    }

    // the cell scan with `extra` leading blocks (overflow carries and step totals) before the scan blocks
    void launch_scan(const Args<R>& A, int extra) {
        const int g = extra + nscan_blocks;
        if (nclouds == 1) {
            if (cell_items == 16) scan_cells<R, CELL_BLOCK, 16, false><<<g, CELL_BLOCK, 0, stream>>>(A);
            else scan_cells<R, CELL_BLOCK, 8, false><<<g, CELL_BLOCK, 0, stream>>>(A);
        } else {
            if (cell_items == 16) scan_cells<R, CELL_BLOCK, 16, true><<<g, CELL_BLOCK, 0, stream>>>(A);
            else scan_cells<R, CELL_BLOCK, 8, true><<<g, CELL_BLOCK, 0, stream>>>(A);
        }
    }

    void enqueue_step(int p) {
        for (int k = 0; k < kNumStepKernels; ++k) launch_step_kernel(k, args[p]);
    }

    // the step sequence of parities p0 (and p1 when >= 0) captured into *out
    void capture_steps(cudaGraphExec_t* out, int p0, int p1) {
        cudaGraph_t g;
        CU(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        enqueue_step(p0);
        if (p1 >= 0) enqueue_step(p1);
        cudaError_t e = cudaStreamEndCapture(stream, &g);
        if (e != cudaSuccess) throw Fail{DSMC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e)};
        e = cudaGraphInstantiate(out, g, 0);
        cudaGraphDestroy(g);
        if (e != cudaSuccess) throw Fail{DSMC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e)};
    }
    void build_graph() {
        if (!graph2) capture_steps(&graph2, 0, 1);
    }
    // one step of parity p: its graph, captured on first use
    void launch_one_step(int p) {
        if (!graph1[p]) capture_steps(&graph1[p], p, -1);
        CU(cudaGraphLaunch(graph1[p], stream));
    }
    void drop_graphs() {
        if (graph2) cudaGraphExecDestroy(graph2);
        graph2 = nullptr;
        for (int p = 0; p < 2; ++p) {
            if (graph1[p]) cudaGraphExecDestroy(graph1[p]);
            graph1[p] = nullptr;
        }
    }

    void step(int n) override {
        if (!initialised) throw Fail{DSMC_ERR_STATE, "dsmc_step before dsmc_init_cloud / dsmc_set_state"};
        if (n < 0) throw Fail{DSMC_ERR_INVALID, "nsteps < 0"};
        int done = 0;
        if (profiling) {
            for (; done < n; ++done) {
                for (int k = 0; k < kNumStepKernels; ++k) {
                    CU(cudaEventRecord(ev[k], stream));
                    launch_step_kernel(k, args[parity]);
                }
                CU(cudaEventRecord(ev[kNumStepKernels], stream));
                CU(cudaEventSynchronize(ev[kNumStepKernels]));
                for (int k = 0; k < kNumStepKernels; ++k) {
                    float ms = 0;
                    CU(cudaEventElapsedTime(&ms, ev[k], ev[k + 1]));
                    prof_ms[k] += ms;
                    prof_n[k] += 1;
                }
                parity ^= 1;
            }
        } else {
            if (use_graphs && n - done >= 2) build_graph();
            if (use_graphs && parity == 1 && n - done >= 1) {
                launch_one_step(1);
                parity = 0;
                ++done;
            }
            while (use_graphs && n - done >= 2) {
                CU(cudaGraphLaunch(graph2, stream));
                done += 2;
            }
            for (; done < n; ++done) {
                if (use_graphs) launch_one_step(parity);
                else enqueue_step(parity);
                parity ^= 1;
            }
        }
        CU(cudaGetLastError());
        steps_taken += n;
    }

    void sync() override { CU(cudaStreamSynchronize(stream)); }

    void set_stream(cudaStream_t s) override {
        sync();
        drop_graphs();
        if (own_stream && stream) cudaStreamDestroy(stream);
        own_stream = false;
        stream = s;
    }

    // ------------------------------------------------------------------ init + full sort
    // Sorts ps/vs/ss (atoms grouped by cloud, counts[k] per cloud) into buffer set 0. The cell
    // scan runs with parity 1 as "current" (zero atoms, zero old starts) so that its "next"
    // outputs land in set 0; then measures the sorted state.
    void sort_and_measure(const R4* ps, const R4* vs, const R4* ss, const std::vector<int>& counts) {
        int n = 0;
        std::vector<int> off(nclouds + 1, 0);
        for (int k = 0; k < nclouds; ++k) { off[k] = n; n += counts[k]; }
        off[nclouds] = n;
        CU(cudaMemcpyAsync(sort_off.p, off.data(), (nclouds + 1) * sizeof(int), cudaMemcpyHostToDevice, stream));
        // the sort's scratch lives in the step's sort keys and mover records (2 and 4 ints per atom
        // of capacity; the keys hold at least 4096 ints), which no sort kernel reads and no step
        // keeps across this call, and the incoming-mover list: no allocation here.
        //   mover records: cell ids | radix keys | radix values (two ping-pong pairs)
        //   sort keys: the digit count table of a pass and its scan's block sums
        //   in_list: the sorted order (source index of each sorted position)
        int* const mr = reinterpret_cast<int*>(mrec.p);
        int* const cell = mr + 2 * (size_t)capacity;
        int* const rkey[2] = {cell, mr};
        int* const rval[2] = {mr + 3 * (size_t)capacity, mr + (size_t)capacity};
        int* const table = reinterpret_cast<int*>(keys.p);
        const int64_t tsize = radix_table(n);
        int* const gb = table + tsize;
        const int tblocks = (int)((tsize + SCAN_CHUNK - 1) / SCAN_CHUNK);
        // reset bookkeeping: parity 1 is "current" with zero atoms, old starts all zero
        CU(cudaMemsetAsync(ctl.p, 0, sizeof(Ctl), stream));
        CU(cudaMemsetAsync(start[1].p, 0, (total_cells + 1) * sizeof(int), stream));
        CU(cudaMemsetAsync(Lc.p, 0, total_cells * sizeof(int), stream));
        CU(cudaMemsetAsync(Ic.p, 0, total_cells * sizeof(int), stream));
        CU(cudaMemsetAsync(cloud_lost.p, 0, nclouds * sizeof(int), stream));
        // the scan's epoch restarts at 0 with the cleared control block: clear its descriptors too
        CU(cudaMemsetAsync(scan_desc.p, 0, (size_t)nscan_blocks * LB_STRIDE * sizeof(unsigned long long), stream));
        Args<R> A = args[1];
        A.init_mode = 1;
        SortArgs<R> S;
        S.pos_src = ps; S.vel_src = vs; S.psi_src = ss;
        S.pos_dst = pos[0].p; S.vel_dst = vel[0].p; S.psi_dst = psi[0].p;
        S.cloud_atom_off = sort_off.p;
        S.cell = cell; S.order = in_list.p;
        S.n = n; S.nclouds = nclouds;
        const int ab = (n + 255) / 256;
        if (n > 0) fs_cells<R><<<ab, 256, 0, stream>>>(S, A);
        launch_scan(A, 0);
        if (cell_items == 16) init_tiles<R, CELL_BLOCK, 16><<<nscan_blocks, CELL_BLOCK, 0, stream>>>(A);
        else init_tiles<R, CELL_BLOCK, 8><<<nscan_blocks, CELL_BLOCK, 0, stream>>>(A);
        if (n > 0) {
            // stable by (cell, source index): LSD passes over the digits of the cell ids
            const int nch = radix_chunks(n), passes = radix_passes(total_cells);
            for (int q = 0; q < passes; ++q) {
                const bool last = q + 1 == passes;
                radix_hist<<<nch, RADIX_BLOCK, 0, stream>>>(rkey[q & 1], n, RADIX_BITS * q, table, nch);
                gscan_reduce<<<tblocks, SCAN_BLOCK, 0, stream>>>(table, (int)tsize, gb);
                gscan_top<<<1, 1024, 0, stream>>>(gb, tblocks, nullptr);
                gscan_down<<<tblocks, SCAN_BLOCK, 0, stream>>>(table, (int)tsize, gb, table);
                radix_scatter<<<nch, RADIX_BLOCK, 0, stream>>>(rkey[q & 1], q == 0 ? nullptr : rval[q & 1], n,
                                                               RADIX_BITS * q, table, nch,
                                                               last ? nullptr : rkey[(q + 1) & 1],
                                                               last ? in_list.p : rval[(q + 1) & 1]);
            }
            fs_gather<R><<<ab, 256, 0, stream>>>(S);
            fill_identity<<<ab, 256, 0, stream>>>(src[0].p, n);
        }
        CU(cudaGetLastError());
        parity = 0;
        // step counter and diagnostics of the sorted state
        measure_tiles<R, 256><<<tile_grid(resident_measure), 256, 0, stream>>>(args[0]);
        finalize<R, true><<<nclouds, 32, 0, stream>>>(args[0]);
        CU(cudaGetLastError());
        CU(cudaStreamSynchronize(stream));
        initialised = true;
        steps_taken = 0;
        check_err();
    }

    void init(uint64_t seed) override {
        run.seed = seed;
        for (int p = 0; p < 2; ++p) args[p].seed = seed;
        sync();
        drop_graphs();  // the step graphs hold the kernel parameters, the seed among them
        int n = 0;
        std::vector<int> off(nclouds + 1, 0), modes(nclouds);
        for (int k = 0; k < nclouds; ++k) {
            off[k] = n;
            n += cloud_atoms_init[k];
            modes[k] = cp[k].init_mode;
        }
        off[nclouds] = n;
        // per-cloud tables in the handle's small buffers (no allocation per call)
        CU(cudaMemcpyAsync(sort_off.p, off.data(), (nclouds + 1) * sizeof(int), cudaMemcpyHostToDevice, stream));
        CU(cudaMemcpyAsync(init_modes.p, modes.data(), nclouds * sizeof(int), cudaMemcpyHostToDevice, stream));
        CU(cudaMemsetAsync(ctl.p, 0, sizeof(Ctl), stream));
        if (n > 0)
            init_atoms<R><<<(n + 255) / 256, 256, 0, stream>>>(args[0], sort_off.p, n, init_modes.p, pos[1].p,
                                                                vel[1].p, psi[1].p, (unsigned long long)seed);
        // (sigma v_r)max per cell
        std::vector<R> sv(nclouds);
        for (int k = 0; k < nclouds; ++k) sv[k] = (R)default_sigvrmax(run, cp[k]);
        CU(cudaMemcpyAsync(init_sv.p, sv.data(), nclouds * sizeof(R), cudaMemcpyHostToDevice, stream));
        fill_sigvrmax<R><<<(total_cells + 255) / 256, 256, 0, stream>>>(sigvrmax.p, d_cell_base.p, init_sv.p, nclouds,
                                                                          total_cells);
        CU(cudaGetLastError());
        sort_and_measure(pos[1].p, vel[1].p, psi[1].p, cloud_atoms_init);
    }

    void check_err() {
        Ctl h;
        CU(cudaMemcpyAsync(&h, ctl.p, sizeof(Ctl), cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        if (h.err) {
            std::string m = "device error bits 0x" + std::to_string(h.err) + ":";
            dsmc_status st = DSMC_ERR_CUDA;
            if (h.err & EB_CELL_FULL) { m += " a tile holds more atoms than it can stage;"; st = DSMC_ERR_CELL_FULL; }
            if (h.err & EB_NAN) { m += " non-finite velocity;"; st = DSMC_ERR_NAN; }
            if (h.err & EB_INIT_REJECT) { m += " initial rejection sampling gave up;"; st = DSMC_ERR_INVALID; }
            if (h.err & EB_TILE_OVERFLOW) { m += " tile table overflow;"; st = DSMC_ERR_CAPACITY; }
            if (h.err & EB_CAPACITY) { m += " a mover or dense-cell list overflowed;"; st = DSMC_ERR_CAPACITY; }
            if (h.err & EB_LOG_FULL) { m += " the collision record is full;"; st = DSMC_ERR_CAPACITY; }
            if (h.err & EB_TIMEOUT) { m += " a bounded device-side wait gave up;"; st = DSMC_ERR_TIMEOUT; }
            if (h.err & EB_INCONSISTENT) { m += " inconsistent cell bookkeeping (after an earlier error);"; }
            throw Fail{st, m};
        }
    }

    // ------------------------------------------------------------------ diagnostics / state
    void diag(int cloud, dsmc_diag* out) override {
        if (!initialised) throw Fail{DSMC_ERR_STATE, "diagnostics before init"};
        if (cloud < -1 || cloud >= nclouds) throw Fail{DSMC_ERR_INVALID, "cloud index out of range"};
        std::vector<CloudDiagDev> g(nclouds);
        CU(cudaMemcpyAsync(g.data(), cdiag.p, nclouds * sizeof(CloudDiagDev), cudaMemcpyDeviceToHost, stream));
        int err = 0;
        CU(cudaMemcpyAsync(&err, &ctl.p->err, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        CU(cudaGetLastError());
        diag_from(g.data(), err, cloud, out);
    }

    // Diagnostics read back without waiting: each slot of a pinned host ring holds one copy of
    // every cloud's step totals and the error bits, taken on the stream when it is enqueued; a
    // collect waits for that copy only (so K steps with a read-back each need not stop the stream).
    // A slot is the clouds' totals (at the slot's 64-byte aligned start: they hold 128-bit sums),
    // then this trailer.
    struct DiagSlotTrailer { int err; int used; };
    unsigned char* diag_host = nullptr;
    std::vector<cudaEvent_t> diag_ev;
    size_t diag_slot_bytes() const {
        return ((nclouds * sizeof(CloudDiagDev) + sizeof(DiagSlotTrailer) + 63) / 64) * 64;
    }
    void free_diag_slots() {
        for (cudaEvent_t e : diag_ev) cudaEventDestroy(e);
        diag_ev.clear();
        if (diag_host) cudaFreeHost(diag_host);
        diag_host = nullptr;
    }
    void diag_reserve(int nslots) override {
        if (nslots < 1 || nslots > (1 << 16)) throw Fail{DSMC_ERR_INVALID, "diagnostics slots must be in [1, 65536]"};
        if ((int)diag_ev.size() >= nslots) return;
        sync();
        free_diag_slots();
        CU(cudaHostAlloc((void**)&diag_host, (size_t)nslots * diag_slot_bytes(), cudaHostAllocDefault));
        memset(diag_host, 0, (size_t)nslots * diag_slot_bytes());
        diag_ev.resize(nslots);
        for (auto& e : diag_ev) CU(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    }
    int64_t diag_copy_bytes() const override { return (int64_t)(nclouds * sizeof(CloudDiagDev) + sizeof(int)); }
    CloudDiagDev* diag_slot(int slot) {
        return reinterpret_cast<CloudDiagDev*>(diag_host + (size_t)slot * diag_slot_bytes());
    }
    DiagSlotTrailer* diag_trailer(int slot) { return reinterpret_cast<DiagSlotTrailer*>(diag_slot(slot) + nclouds); }
    void diag_enqueue(int slot) override {
        if (!initialised) throw Fail{DSMC_ERR_STATE, "diagnostics before init"};
        if (slot < 0 || slot >= (int)diag_ev.size()) throw Fail{DSMC_ERR_INVALID, "diagnostics slot not reserved"};
        DiagSlotTrailer* tr = diag_trailer(slot);
        CU(cudaMemcpyAsync(diag_slot(slot), cdiag.p, nclouds * sizeof(CloudDiagDev), cudaMemcpyDeviceToHost, stream));
        CU(cudaMemcpyAsync(&tr->err, &ctl.p->err, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CU(cudaEventRecord(diag_ev[slot], stream));
        tr->used = 1;
    }
    void diag_collect(int slot, int cloud, dsmc_diag* out) override {
        if (slot < 0 || slot >= (int)diag_ev.size()) throw Fail{DSMC_ERR_INVALID, "diagnostics slot not reserved"};
        if (cloud < -1 || cloud >= nclouds) throw Fail{DSMC_ERR_INVALID, "cloud index out of range"};
        const DiagSlotTrailer* tr = diag_trailer(slot);
        if (!tr->used) throw Fail{DSMC_ERR_STATE, "diagnostics slot collected before it was enqueued"};
        CU(cudaEventSynchronize(diag_ev[slot]));
        diag_from(diag_slot(slot), tr->err, cloud, out);
    }

    // the diagnostics of `cloud` (-1: all) from a copy of the clouds' step totals
    void diag_from(const CloudDiagDev* g, int ctl_err, int cloud, dsmc_diag* out) {
        int k0 = cloud < 0 ? 0 : cloud, k1 = cloud < 0 ? nclouds : cloud + 1;
        CloudDiagDev s;
        memset(&s, 0, sizeof(s));
        double e_kin = 0, e_pot = 0, e_evap = 0;
        double msum = 0;
        int err = 0;
        for (int k = k0; k < k1; ++k) {
            const CloudDiagDev& d = g[k];
            const CloudPhys<R>& P = phys[k];
            s.step = d.step;
            s.n_alive += d.n_alive;
            s.sum_v2 += d.sum_v2;
            s.sum_B += d.sum_B;
            s.cum_evap += d.cum_evap; s.cum_maj += d.cum_maj; s.cum_knife += d.cum_knife;
            s.cum_coll += d.cum_coll; s.cum_cand += d.cum_cand;
            s.cum_atom_steps += d.cum_atom_steps;
            e_kin += 0.5 * P.mass * fx_to_double(d.sum_v2);
            e_pot += P.moment * fx_to_double(d.sum_B);
            e_evap += 0.5 * P.mass * fx_to_double(d.cum_evap_v2) + P.moment * fx_to_double(d.cum_evap_B);
            msum += P.mass * fx_to_double(d.sum_v2);
            err |= (int)d.err;
        }
        memset(out, 0, sizeof(*out));
        out->step = s.step;
        out->time = (double)s.step * run.dt;
        out->n_alive = s.n_alive;
        out->e_kin = e_kin;
        out->e_pot = e_pot;
        out->sum_v2 = fx_to_double(s.sum_v2);
        out->sum_absB = fx_to_double(s.sum_B);
        out->temperature = s.n_alive > 0 ? msum / (3.0 * phys[k0].kB * (double)s.n_alive) : 0.0;
        out->n_evaporated = s.cum_evap;
        out->n_majorana = s.cum_maj;
        out->n_knife = s.cum_knife;
        out->e_evaporated = e_evap;
        out->collisions = s.cum_coll;
        out->candidates = s.cum_cand;
        out->atom_steps = s.cum_atom_steps;
        out->error = ctl_err | err;
    }

    void get_state(dsmc_state_buffers* o) override {
        if (!initialised) throw Fail{DSMC_ERR_STATE, "get_state before init"};
        sync();
        Ctl h;
        CU(cudaMemcpy(&h, ctl.p, sizeof(Ctl), cudaMemcpyDeviceToHost));
        const int n = h.n[parity];
        if (o->n < n) throw Fail{DSMC_ERR_INVALID, "state buffers too small: need " + std::to_string(n)};
        std::vector<CloudDyn> d(nclouds);
        CU(cudaMemcpy(d.data(), cdyn.p, nclouds * sizeof(CloudDyn), cudaMemcpyDeviceToHost));
        // the state is stored in the order of the previous step; gather it into sorted order in
        // the other buffer set (free between steps) and copy that
        const int q = 1 - parity;
        if (n > 0)
            materialize<R><<<(n + 255) / 256, 256, 0, stream>>>(args[parity], n, pos[q].p, vel[q].p, psi[q].p);
        CU(cudaGetLastError());
        if (o->pos) CU(cudaMemcpyAsync(o->pos, pos[q].p, (size_t)n * sizeof(R4), cudaMemcpyDeviceToHost, stream));
        if (o->vel) CU(cudaMemcpyAsync(o->vel, vel[q].p, (size_t)n * sizeof(R4), cudaMemcpyDeviceToHost, stream));
        if (o->psi) CU(cudaMemcpyAsync(o->psi, psi[q].p, (size_t)n * sizeof(R4), cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        o->n = n;
        if (o->cloud_counts)
            for (int k = 0; k < nclouds; ++k) o->cloud_counts[k] = d[k].n[parity];
    }

    void set_state(const dsmc_state_buffers* in) override {
        if (!in || !in->pos || !in->vel || !in->psi || !in->cloud_counts)
            throw Fail{DSMC_ERR_INVALID, "set_state needs pos, vel, psi and cloud_counts"};
        std::vector<int> counts(nclouds);
        int64_t tot = 0;
        for (int k = 0; k < nclouds; ++k) {
            if (in->cloud_counts[k] < 0) throw Fail{DSMC_ERR_INVALID, "negative cloud count"};
            counts[k] = (int)in->cloud_counts[k];
            tot += in->cloud_counts[k];
        }
        if (tot != in->n) throw Fail{DSMC_ERR_INVALID, "cloud_counts do not add up to n"};
        if (tot > capacity) throw Fail{DSMC_ERR_CAPACITY, "more atoms than the handle's capacity"};
        CU(cudaMemcpyAsync(pos[1].p, in->pos, (size_t)tot * sizeof(R4), cudaMemcpyHostToDevice, stream));
        CU(cudaMemcpyAsync(vel[1].p, in->vel, (size_t)tot * sizeof(R4), cudaMemcpyHostToDevice, stream));
        CU(cudaMemcpyAsync(psi[1].p, in->psi, (size_t)tot * sizeof(R4), cudaMemcpyHostToDevice, stream));
        if (!initialised) {
            // sigvrmax defaults as at init
            std::vector<R> sv(total_cells);
            for (int k = 0; k < nclouds; ++k) {
                const R v = (R)default_sigvrmax(run, cp[k]);
                for (int cc = cloud_cell_base[k]; cc < cloud_cell_base[k + 1]; ++cc) sv[cc] = v;
            }
            CU(cudaMemcpyAsync(sigvrmax.p, sv.data(), total_cells * sizeof(R), cudaMemcpyHostToDevice, stream));
            CU(cudaStreamSynchronize(stream));
        }
        sort_and_measure(pos[1].p, vel[1].p, psi[1].p, counts);
    }

    void get_cell_starts(int32_t* st, int64_t cap, int64_t* total) override {
        if (total) *total = total_cells;
        if (!st) return;
        if (cap < total_cells + 1) throw Fail{DSMC_ERR_INVALID, "cell start buffer too small"};
        sync();
        CU(cudaMemcpy(st, start[parity].p, (total_cells + 1) * sizeof(int), cudaMemcpyDeviceToHost));
    }

    void get_sigvrmax(void* out, int64_t cap) override {
        if (cap < total_cells) throw Fail{DSMC_ERR_INVALID, "sigvrmax buffer too small"};
        sync();
        CU(cudaMemcpy(out, sigvrmax.p, total_cells * sizeof(R), cudaMemcpyDeviceToHost));
    }
    void set_sigvrmax(const void* in, int64_t n) override {
        if (n != total_cells) throw Fail{DSMC_ERR_INVALID, "sigvrmax length must equal the number of cells"};
        sync();
        CU(cudaMemcpy(sigvrmax.p, in, total_cells * sizeof(R), cudaMemcpyHostToDevice));
    }

    // The coming step's scan on its own, its ticket counter started at 1: no block processes scan
    // block 0, whose descriptor therefore never appears in this launch, and the blocks looking
    // back to it give up after their time limit. The scan reads the current starts and the
    // (cleared) leaver / incoming counters and writes only the coming step's starts, tiles and
    // counters, which the next step's scan writes again; the extra blocks (step totals, overflow
    // carries) are left out of the launch.
    int check_wait_timeout() override {
        if (!initialised) throw Fail{DSMC_ERR_STATE, "wait check before init"};
        if (nscan_blocks < 2) throw Fail{DSMC_ERR_INVALID, "the wait check needs more than one scan block of cells"};
        sync();
        check_err();
        // the dense-cell lists: the scan lists into one and clears the other, which the coming
        // step's dense_collide still reads, so both are put back afterwards
        int nd[2] = {0, 0};
        CU(cudaMemcpyAsync(nd, ctl.p->ndense, sizeof(nd), cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        const int one = 1;
        CU(cudaMemcpyAsync(&ctl.p->scan_ticket, &one, sizeof(int), cudaMemcpyHostToDevice, stream));
        launch_scan(args[parity], 0);
        CU(cudaGetLastError());
        int bits = 0;
        CU(cudaMemcpyAsync(&bits, &ctl.p->err, sizeof(int), cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        CU(cudaMemsetAsync(&ctl.p->err, 0, sizeof(int), stream));
        CU(cudaMemcpyAsync(ctl.p->ndense, nd, sizeof(nd), cudaMemcpyHostToDevice, stream));
        CU(cudaStreamSynchronize(stream));
        return bits;
    }

    void set_profiling(bool on) override {
        profiling = on;
        for (int k = 0; k < kNumStepKernels; ++k) { prof_ms[k] = 0; prof_n[k] = 0; }
    }
    // Times dsmc_step with each candidate launch shape (nominal tile size x step-kernel blocks per
    // SM; the simulation advances meanwhile; results do not depend on the shape) and keeps the
    // fastest.  A new tile size takes effect one step after it is set (the tiling of a step is
    // built by the scan of the step before).
    std::vector<int> tune_T, tune_B;
    std::vector<double> tune_ms;
    void autotune(int steps_per_candidate, int32_t* chosen, double* ms_per_step) override {
        if (!initialised) throw Fail{DSMC_ERR_STATE, "autotune before init"};
        if (steps_per_candidate < 1) throw Fail{DSMC_ERR_INVALID, "steps_per_candidate must be >= 1"};
        const int cands[] = {128, 192, 240, 256, 384, 448, 480, 496, 512, CAP - BLOCK - 16, 768, 960, 1024};
        int best = tile_nominal, best_b = step_bps;
        double best_ms = 1e300;
        const bool prof = profiling;
        profiling = false;
        tune_T.clear(); tune_B.clear(); tune_ms.clear();
        for (int bps = step_occ; bps >= 1 && bps >= step_occ - 2; --bps) {
            for (int T : cands) {
                if (T > CAP - 128) continue;
                set_shape(T, bps);
                step(1);  // builds the tiling of size T
                CU(cudaEventRecord(ev[0], stream));
                step(steps_per_candidate);
                CU(cudaEventRecord(ev[1], stream));
                CU(cudaEventSynchronize(ev[1]));
                float ms = 0;
                CU(cudaEventElapsedTime(&ms, ev[0], ev[1]));
                const double per = ms / steps_per_candidate;
                tune_T.push_back(T); tune_B.push_back(bps); tune_ms.push_back(per);
                if (per < best_ms) { best_ms = per; best = T; best_b = bps; }
            }
        }
        set_shape(best, best_b);
        step(1);
        profiling = prof;
        check_err();
        if (chosen) *chosen = best;
        if (ms_per_step) *ms_per_step = best_ms;
    }
    void autotune_table(int32_t* T, int32_t* B, double* ms, int cap, int32_t* count, int32_t* chosen_b) override {
        const int n = (int)tune_T.size();
        for (int i = 0; i < std::min(n, cap); ++i) {
            if (T) T[i] = tune_T[i];
            if (B) B[i] = tune_B[i];
            if (ms) ms[i] = tune_ms[i];
        }
        if (count) *count = n;
        if (chosen_b) *chosen_b = step_bps;
    }

    // a launch shape: nominal tile size T and step-kernel blocks per SM
    void set_shape(int T, int bps) {
        step_bps = std::max(1, std::min(bps, step_occ));
        resident_step = num_sms * step_bps;
        set_tile(T);
    }

    void set_tile(int T) {
        sync();
        tile_nominal = T;
        for (int p = 0; p < 2; ++p) {
            args[p].tile_nominal = T;
            args[p].tile_fill = 0;  // a chosen size is kept as given
        }
        drop_graphs();
    }

    // ------------------------------------------------------------------ adjoint
    // record: the physical run's initial state by atom id and its collision events
    DevBuf<double> adj_x0, adj_v0, adj_p0, adj_n, adj_sums, adj_theta_b;
    DevBuf<int2> adj_ij;
    DevBuf<int> adj_off, adj_count;
    int adj_steps = -1, adj_natoms = 0, adj_nlog = 0, adj_K = 100, adj_prec = DSMC_FP64;
    double adj_width = 0.2, adj_maj_width = 0.05;

    void adjoint_run(const dsmc_adj_params* ap, dsmc_grad* g) override {
        if (!initialised) throw Fail{DSMC_ERR_STATE, "adjoint before init"};
        if (nclouds != 1 || cp[0].trap != DSMC_TRAP_QUADRUPOLE)
            throw Fail{DSMC_ERR_UNSUPPORTED, "the adjoint supports one cloud in the linear (quadrupole) trap"};
        if (steps_taken != 0) throw Fail{DSMC_ERR_STATE, "call dsmc_adjoint_run right after dsmc_init_cloud"};
        if (ap->steps < 1 || ap->checkpoint_every < 1 || !(ap->sigmoid_width_kT > 0))
            throw Fail{DSMC_ERR_INVALID, "adjoint: steps, checkpoint_every and sigmoid_width_kT must be positive"};
        if (ap->precision != DSMC_FP32 && ap->precision != DSMC_FP64) throw Fail{DSMC_ERR_INVALID, "adjoint precision"};
        sync();
        Ctl h;
        CU(cudaMemcpy(&h, ctl.p, sizeof(Ctl), cudaMemcpyDeviceToHost));
        const int n = h.n[parity];
        if (n != (int)cp[0].n_atoms) throw Fail{DSMC_ERR_STATE, "adjoint: atoms were lost before the run"};
        adj_steps = ap->steps; adj_natoms = n; adj_K = ap->checkpoint_every; adj_prec = ap->precision;
        adj_width = ap->sigmoid_width_kT;
        adj_maj_width = ap->majorana_width > 0 ? ap->majorana_width : 0.05;
        adj_x0.alloc(3 * (size_t)std::max(n, 1)); adj_v0.alloc(3 * (size_t)std::max(n, 1));
        adj_p0.alloc(4 * (size_t)std::max(n, 1));
        if (n > 0)
            state_by_id<R><<<(n + 255) / 256, 256, 0, stream>>>(args[parity], n, adj_x0.p, adj_v0.p, adj_p0.p,
                                                                 &ctl.p->err);
        const int cap = 1 << 22;
        adj_ij.alloc(cap); adj_n.alloc(3 * (size_t)cap); adj_off.alloc(ap->steps + 1); adj_count.alloc(1);
        CU(cudaMemsetAsync(adj_off.p, 0, (ap->steps + 1) * sizeof(int), stream));
        CU(cudaMemsetAsync(adj_count.p, 0, sizeof(int), stream));
        // the physical run, recording every accepted collision
        for (int p = 0; p < 2; ++p) {
            args[p].clog_ij = adj_ij.p; args[p].clog_n = adj_n.p; args[p].clog_count = adj_count.p;
            args[p].clog_off = adj_off.p; args[p].clog_cap = cap; args[p].clog_step0 = 0;
            args[p].clog_steps = ap->steps;
        }
        drop_graphs();
        cudaEvent_t e0 = ev[0], e1 = ev[1];
        CU(cudaEventRecord(e0, stream));
        step(ap->steps);
        CU(cudaEventRecord(e1, stream));
        CU(cudaEventSynchronize(e1));
        float ms_rec = 0;
        CU(cudaEventElapsedTime(&ms_rec, e0, e1));
        for (int p = 0; p < 2; ++p) {
            args[p].clog_ij = nullptr; args[p].clog_n = nullptr; args[p].clog_count = nullptr;
            args[p].clog_off = nullptr; args[p].clog_cap = 0;
        }
        drop_graphs();
        check_err();
        int cnt = 0;
        CU(cudaMemcpy(&cnt, adj_count.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (cnt > cap) throw Fail{DSMC_ERR_CAPACITY, "adjoint: more than 2^22 collisions recorded; run fewer steps"};
        adj_nlog = cnt;
        // the smoothed model at the run's own parameters, forward and backward
        double theta[ADJ_NPARAM];
        own_theta(theta);
        double parts[2] = {0, 0}, tb[ADJ_SEEDS * ADJ_NPARAM] = {0}, ms_f = 0, ms_b = 0;
        smoothed(theta, true, parts, tb, &ms_f, &ms_b);
        memset(g, 0, sizeof(*g));
        g->loss = parts[0] + parts[1];
        g->mean_energy_kT = parts[0];
        g->retained_fraction = parts[1];
        for (int k = 0; k < ADJ_NPARAM; ++k) {
            g->dE_dtheta[k] = tb[k];
            g->dN_dtheta[k] = tb[ADJ_NPARAM + k];
        }
        g->dL_dBp = tb[0] + tb[ADJ_NPARAM];
        g->dL_dB0 = tb[1] + tb[ADJ_NPARAM + 1];
        for (int k = 0; k < 9; ++k) g->dL_deta[k] = tb[2 + k] + tb[ADJ_NPARAM + 2 + k];
        g->collisions = adj_nlog;
        g->ms_record = ms_rec;
        g->ms_forward = ms_f;
        g->ms_backward = ms_b;
    }

    void own_theta(double* theta) const {
        theta[0] = cp[0].dBdz;
        theta[1] = cp[0].B0;
        for (int k = 0; k < 9; ++k) theta[2 + k] = cp[0].knife_eta[k];
    }

    // the smoothed loss terms parts = (L_E, L_N) at theta and, with grad, their gradients in tb
    // (ADJ_SEEDS x ADJ_NPARAM: d L_E, then d L_N)
    void smoothed(const double* theta, bool grad, double* parts, double* tb, double* ms_f, double* ms_b) {
        if (adj_prec == DSMC_FP64) smoothed_t<double>(theta, grad, parts, tb, ms_f, ms_b);
        else smoothed_t<float>(theta, grad, parts, tb, ms_f, ms_b);
    }

    template <class S>
    void smoothed_t(const double* theta, bool grad, double* parts, double* tb, double* ms_f, double* ms_b) {
        typedef typename V4T<S>::type S4;
        const int n = adj_natoms, steps = adj_steps, K = adj_K;
        const dsmc_cloud_params& c = cp[0];
        const double kB = phys[0].kB;
        SmoothArgs<S> A;
        memset(&A, 0, sizeof(A));
        A.C.Bp = (S)theta[0];
        A.C.B0 = (S)theta[1];
        A.C.B_floor = (S)0;
        A.C.dt = (S)run.dt;
        A.C.half_dt = (S)(0.5 * run.dt);
        A.C.accel_scale = (S)(c.moment / c.mass);
        A.C.kappa = (S)(2.0 * c.moment / c.mass);
        A.C.inv_width = (S)(1.0 / (2.0 * adj_width * kB * c.temperature / c.mass));
        A.C.theta_per_B = (c.flags & DSMC_F_LARMOR) ? (S)(c.moment * run.dt / run_hbar(run)) : (S)0;
        A.C.inv_width_maj = (c.flags & DSMC_F_MAJORANA) ? (S)(1.0 / adj_maj_width) : (S)0;
        A.C.cut_scale = 2.0 * kB * c.temperature / c.mass;
        A.n = n;
        const int nn = std::max(n, 1);
        DevBuf<S4> x, v, ps, xb, vb, pb, vpre, seg_x, seg_v, seg_p, ck_x, ck_v, ck_p;
        DevBuf<S> e;  // the survival weight rides in x's fourth lane, its adjoints in xb's
        x.alloc(nn); v.alloc(nn); ps.alloc(nn); e.alloc(nn);
        const int nseg = (steps + K - 1) / K;
        const int ab = (nn + 255) / 256;
        const int sum_blocks = std::min(ab, 1184);
        int occ = 0;
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, sm_move<S>, 256, 0));
        const int move_blocks = std::min(ab, num_sms * std::max(occ, 1));
        CU(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, adj_move<S>, 256, 0));
        const int adj_blocks = std::min(ab, num_sms * std::max(occ, 1));
        partials_buf.alloc(sum_blocks);
        adj_sums.alloc(2);
        DevBuf<int> done;
        done.alloc(1);
        CU(cudaMemsetAsync(done.p, 0, sizeof(int), stream));
        A.x = x.p; A.v = v.p; A.psi = ps.p; A.e = e.p;
        A.ij = adj_ij.p; A.nv = adj_n.p; A.off = adj_off.p; A.partials = partials_buf.p;
        A.done = done.p;
        DevBuf<double> theta_part;
        if (grad) {
            vpre.alloc(2 * (size_t)std::max(adj_nlog, 1));
            seg_x.alloc((size_t)K * nn); seg_v.alloc((size_t)K * nn); seg_p.alloc((size_t)K * nn);
            ck_x.alloc((size_t)nseg * nn); ck_v.alloc((size_t)nseg * nn); ck_p.alloc((size_t)nseg * nn);
            xb.alloc(ADJ_SEEDS * (size_t)nn); vb.alloc(ADJ_SEEDS * (size_t)nn); pb.alloc(ADJ_SEEDS * (size_t)nn);
            adj_theta_b.alloc(ADJ_SEEDS * ADJ_NPARAM);
            CU(cudaMemsetAsync(adj_theta_b.p, 0, ADJ_SEEDS * ADJ_NPARAM * sizeof(double), stream));
            theta_part.alloc((size_t)adj_blocks * ADJ_SEEDS * ADJ_NPARAM);
            CU(cudaMemsetAsync(theta_part.p, 0, (size_t)adj_blocks * ADJ_SEEDS * ADJ_NPARAM * sizeof(double), stream));
            A.theta_part = theta_part.p;
            A.vpre = vpre.p; A.seg_x = seg_x.p; A.seg_v = seg_v.p; A.seg_psi = seg_p.p;
            A.xb = xb.p; A.vb = vb.p; A.pb = pb.p; A.theta_b = adj_theta_b.p;
        }
        std::vector<S> cuts(steps);
        for (int t = 0; t < steps; ++t)
            cuts[t] = (S)(A.C.cut_scale * knife_eta(c.knife_nknots, c.knife_step, theta + 2, (double)t));
        CU(cudaEventRecord(ev[0], stream));
        if (n > 0) sm_load<S><<<ab, 256, 0, stream>>>(A, adj_x0.p, adj_v0.p, adj_p0.p);
        // a step is one launch: the move, then the next step's collisions in its last block -- except
        // before a checkpoint, which keeps the state the next step starts from before its collisions
        for (int t = 0; n > 0 && t < steps; ++t) {
            const bool ck = grad && t % K == 0;
            if (ck) {
                const size_t o = (size_t)(t / K) * nn;
                CU(cudaMemcpyAsync(ck_x.p + o, x.p, n * sizeof(S4), cudaMemcpyDeviceToDevice, stream));
                CU(cudaMemcpyAsync(ck_v.p + o, v.p, n * sizeof(S4), cudaMemcpyDeviceToDevice, stream));
                CU(cudaMemcpyAsync(ck_p.p + o, ps.p, n * sizeof(S4), cudaMemcpyDeviceToDevice, stream));
            }
            if (t == 0 || ck) sm_collide<S><<<1, 32, 0, stream>>>(A, t, 0, -1);
            const bool fuse = t + 1 < steps && !(grad && (t + 1) % K == 0);
            sm_move<S><<<move_blocks, 256, 0, stream>>>(A, cuts[t], -1, t == steps - 1 ? 1 : 0, fuse ? t + 1 : -1, 0);
        }
        if (n > 0) sm_sums<S><<<sum_blocks, 256, 0, stream>>>(A);
        sm_sums_final<<<1, 32, 0, stream>>>(partials_buf.p, n > 0 ? sum_blocks : 0, adj_sums.p);
        CU(cudaEventRecord(ev[1], stream));
        double sums[2];
        CU(cudaMemcpyAsync(sums, adj_sums.p, 2 * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        float mf = 0;
        CU(cudaEventElapsedTime(&mf, ev[0], ev[1]));
        if (ms_f) *ms_f = mf;
        const double kT = kB * c.temperature;
        const double Wd = sums[0], Sd = sums[1];
        parts[0] = 0.5 * c.mass * Sd / Wd / kT;
        parts[1] = Wd / (double)n;
        CU(cudaGetLastError());
        if (!grad) return;
        CU(cudaEventRecord(ev[2], stream));
        const double half_m_over_kT = 0.5 * c.mass / kT;
        if (n > 0) adj_seed<S><<<adj_blocks, 256, 0, stream>>>(A, adj_sums.p, half_m_over_kT);
        for (int s = nseg - 1; n > 0 && s >= 0; --s) {
            const int t0 = s * K, t1 = std::min(steps, t0 + K);
            const size_t o = (size_t)s * nn;
            // the segment from its checkpoint, slot to slot: slot t - t0 holds the state step t starts
            // from (after its collisions), which is all the adjoint steps read
            CU(cudaMemcpyAsync(seg_x.p, ck_x.p + o, n * sizeof(S4), cudaMemcpyDeviceToDevice, stream));
            CU(cudaMemcpyAsync(seg_v.p, ck_v.p + o, n * sizeof(S4), cudaMemcpyDeviceToDevice, stream));
            CU(cudaMemcpyAsync(seg_p.p, ck_p.p + o, n * sizeof(S4), cudaMemcpyDeviceToDevice, stream));
            sm_collide<S><<<1, 32, 0, stream>>>(A, t0, 1, 0);
            for (int t = t0; t + 1 < t1; ++t)
                sm_move<S><<<move_blocks, 256, 0, stream>>>(A, cuts[t], t - t0, 0, t + 1, 1);
            for (int t = t1 - 1; t >= t0; --t) {
                int k0 = 0;
                double f = 0;
                knot_weights(c.knife_nknots, c.knife_step, (double)t, &k0, &f);
                adj_move<S><<<adj_blocks, 256, 0, stream>>>(A, cuts[t], t - t0, k0, f, t);
            }
        }
        adj_theta_reduce<<<1, 32 * ADJ_SEEDS * ADJ_NPARAM, 0, stream>>>(theta_part.p, adj_blocks, adj_theta_b.p);
        CU(cudaEventRecord(ev[3], stream));
        CU(cudaMemcpyAsync(tb, adj_theta_b.p, ADJ_SEEDS * ADJ_NPARAM * sizeof(double), cudaMemcpyDeviceToHost, stream));
        CU(cudaStreamSynchronize(stream));
        CU(cudaGetLastError());
        float mb = 0;
        CU(cudaEventElapsedTime(&mb, ev[2], ev[3]));
        if (ms_b) *ms_b = mb;
    }
    DevBuf<TilePartial> partials_buf;

    void adjoint_loss(const double* theta, double* parts, double* grad_e, double* grad_n) override {
        if (adj_steps < 0) throw Fail{DSMC_ERR_STATE, "dsmc_adjoint_loss needs a recorded run (dsmc_adjoint_run)"};
        double own[ADJ_NPARAM];
        own_theta(own);
        const double* th = theta ? theta : own;
        double tb[ADJ_SEEDS * ADJ_NPARAM] = {0};
        smoothed(th, grad_e != nullptr || grad_n != nullptr, parts, tb, nullptr, nullptr);
        for (int k = 0; k < ADJ_NPARAM; ++k) {
            if (grad_e) grad_e[k] = tb[k];
            if (grad_n) grad_n[k] = tb[ADJ_NPARAM + k];
        }
    }

    // ------------------------------------------------------------------ snapshot records
    DevBuf<R4> rec_pos, rec_vel;
    DevBuf<int2> rec_coll;
    int rec_flags = 0;

    void set_recording(int flags) override {
        if (flags & ~(DSMC_REC_EVAPORATED | DSMC_REC_CELL_COLLISIONS)) throw Fail{DSMC_ERR_INVALID, "unknown record flags"};
        sync();
        if ((flags & DSMC_REC_EVAPORATED) && !rec_pos.p) { rec_pos.alloc(capacity); rec_vel.alloc(capacity); }
        if ((flags & DSMC_REC_CELL_COLLISIONS) && !rec_coll.p) rec_coll.alloc(total_cells);
        // cleared on every call: never lost (step lane all ones), never collided (step -1)
        if (flags & DSMC_REC_EVAPORATED) {
            CU(cudaMemsetAsync(rec_pos.p, 0xff, capacity * sizeof(R4), stream));
            CU(cudaMemsetAsync(rec_vel.p, 0, capacity * sizeof(R4), stream));
        }
        if (flags & DSMC_REC_CELL_COLLISIONS) CU(cudaMemsetAsync(rec_coll.p, 0xff, total_cells * sizeof(int2), stream));
        rec_flags = flags;
        for (int p = 0; p < 2; ++p) {
            args[p].rec_evap_pos = (flags & DSMC_REC_EVAPORATED) ? rec_pos.p : nullptr;
            args[p].rec_evap_vel = (flags & DSMC_REC_EVAPORATED) ? rec_vel.p : nullptr;
            args[p].rec_cell_coll = (flags & DSMC_REC_CELL_COLLISIONS) ? rec_coll.p : nullptr;
        }
        drop_graphs();  // the step graphs hold the kernel parameters
        sync();
    }

    void get_evaporated(int cloud, double* pos3, double* vel3, int32_t* step_out, int32_t* fate, int64_t cap) override {
        if (!(rec_flags & DSMC_REC_EVAPORATED)) throw Fail{DSMC_ERR_STATE, "evaporated atoms are not recorded (dsmc_set_recording)"};
        if (cloud < 0 || cloud >= nclouds) throw Fail{DSMC_ERR_INVALID, "cloud index"};
        const int base = phys[cloud].id_base, n = phys[cloud].id_cap;
        if (cap < n) throw Fail{DSMC_ERR_INVALID, "buffers smaller than the cloud's capacity"};
        sync();
        std::vector<R4> hp(n), hv(n);
        if (n > 0) {
            CU(cudaMemcpy(hp.data(), rec_pos.p + base, n * sizeof(R4), cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(hv.data(), rec_vel.p + base, n * sizeof(R4), cudaMemcpyDeviceToHost));
        }
        for (int i = 0; i < n; ++i) {
            const uint32_t st = lane_to_u32(hp[i].w);
            const bool lost = st != 0xffffffffu;
            if (pos3) { pos3[3 * i] = lost ? (double)hp[i].x : 0.0; pos3[3 * i + 1] = lost ? (double)hp[i].y : 0.0;
                        pos3[3 * i + 2] = lost ? (double)hp[i].z : 0.0; }
            if (vel3) { vel3[3 * i] = (double)hv[i].x; vel3[3 * i + 1] = (double)hv[i].y; vel3[3 * i + 2] = (double)hv[i].z; }
            if (step_out) step_out[i] = lost ? (int32_t)st : -1;
            if (fate) fate[i] = lost ? (int32_t)lane_to_u32(hv[i].w) : 0;
        }
    }

    void get_cell_collisions(int32_t* counts, int64_t cap, int64_t* total) override {
        if (!(rec_flags & DSMC_REC_CELL_COLLISIONS)) throw Fail{DSMC_ERR_STATE, "cell collisions are not recorded (dsmc_set_recording)"};
        if (total) *total = total_cells;
        if (!counts) return;
        if (cap < total_cells) throw Fail{DSMC_ERR_INVALID, "buffer smaller than the cell count"};
        sync();
        Ctl h;
        CU(cudaMemcpy(&h, ctl.p, sizeof(Ctl), cudaMemcpyDeviceToHost));
        // the last step that ran the collisions: the largest s below the coming step with s % collide_every == 0
        const int next = h.step[parity];
        const int last = next > 0 ? ((next - 1) / run.collide_every) * run.collide_every : -1;
        std::vector<int2> hc(total_cells);
        CU(cudaMemcpy(hc.data(), rec_coll.p, total_cells * sizeof(int2), cudaMemcpyDeviceToHost));
        for (int c = 0; c < total_cells; ++c) counts[c] = (last >= 0 && hc[c].x == last) ? hc[c].y : 0;
    }

    void adjoint_export_spinors(double* psi0, int64_t atoms_cap) override {
        if (adj_steps < 0) throw Fail{DSMC_ERR_STATE, "nothing recorded (dsmc_adjoint_run)"};
        if (atoms_cap < adj_natoms) throw Fail{DSMC_ERR_INVALID, "spinor buffer too small"};
        sync();
        CU(cudaMemcpy(psi0, adj_p0.p, 4 * (size_t)adj_natoms * sizeof(double), cudaMemcpyDeviceToHost));
    }

    void adjoint_export(double* x0, double* v0, int64_t atoms_cap, int32_t* off, int64_t off_cap, int32_t* ij,
                        double* nv, int64_t log_cap, int64_t* n_atoms, int64_t* n_log, int32_t* steps_out) override {
        if (adj_steps < 0) throw Fail{DSMC_ERR_STATE, "nothing recorded (dsmc_adjoint_run)"};
        if (n_atoms) *n_atoms = adj_natoms;
        if (n_log) *n_log = adj_nlog;
        if (steps_out) *steps_out = adj_steps;
        sync();
        if (x0 && v0) {
            if (atoms_cap < adj_natoms) throw Fail{DSMC_ERR_INVALID, "atom buffers too small"};
            CU(cudaMemcpy(x0, adj_x0.p, 3 * (size_t)adj_natoms * sizeof(double), cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(v0, adj_v0.p, 3 * (size_t)adj_natoms * sizeof(double), cudaMemcpyDeviceToHost));
        }
        if (off) {
            if (off_cap < adj_steps + 1) throw Fail{DSMC_ERR_INVALID, "offset buffer too small"};
            CU(cudaMemcpy(off, adj_off.p, (adj_steps + 1) * sizeof(int), cudaMemcpyDeviceToHost));
        }
        if (ij && nv) {
            if (log_cap < adj_nlog) throw Fail{DSMC_ERR_INVALID, "record buffers too small"};
            CU(cudaMemcpy(ij, adj_ij.p, 2 * (size_t)adj_nlog * sizeof(int), cudaMemcpyDeviceToHost));
            CU(cudaMemcpy(nv, adj_n.p, 3 * (size_t)adj_nlog * sizeof(double), cudaMemcpyDeviceToHost));
        }
    }

    void kernel_times(const char** names, double* ms, int64_t* launches, int cap, int* count) override {
        const int n = std::min(cap, kNumStepKernels);
        for (int k = 0; k < n; ++k) {
            if (names) names[k] = kKernelNames[k];
            if (ms) ms[k] = prof_ms[k];
            if (launches) launches[k] = prof_n[k];
        }
        if (count) *count = kNumStepKernels;
    }
};

template <class F> dsmc_status guard(dsmc_handle* h, F&& f) {
    try {
        f();
        if (h) h->last_error.clear();
        return DSMC_OK;
    } catch (const Fail& e) {
        if (h) h->last_error = e.msg;
        return e.st;
    } catch (const std::exception& e) {
        if (h) h->last_error = e.what();
        return DSMC_ERR_ALLOC;
    }
}

thread_local std::string g_create_error;

}  // namespace

// ====================================================================================== C ABI
DSMC_API int32_t dsmc_abi_version(void) { return DSMC_ABI_VERSION; }

DSMC_API const char* dsmc_status_string(dsmc_status s) {
    switch (s) {
    case DSMC_OK: return "ok";
    case DSMC_ERR_INVALID: return "invalid argument";
    case DSMC_ERR_CUDA: return "CUDA error";
    case DSMC_ERR_ALLOC: return "allocation failed";
    case DSMC_ERR_CAPACITY: return "capacity exceeded";
    case DSMC_ERR_CELL_FULL: return "tile too full to stage";
    case DSMC_ERR_NAN: return "non-finite state";
    case DSMC_ERR_STATE: return "call out of order";
    case DSMC_ERR_UNSUPPORTED: return "unsupported";
    case DSMC_ERR_TIMEOUT: return "device wait timed out";
    }
    return "unknown status";
}

DSMC_API const char* dsmc_last_error(const dsmc_handle* h) {
    return h ? h->last_error.c_str() : g_create_error.c_str();
}

DSMC_API dsmc_status dsmc_preset(int32_t which, dsmc_params* run, dsmc_cloud_params* c) {
    if (!run || !c) return DSMC_ERR_INVALID;
    return fill_preset(which, run, c);
}

DSMC_API dsmc_status dsmc_create(const dsmc_params* run, const dsmc_cloud_params* clouds, int32_t nclouds,
                                 dsmc_handle** out) {
    g_create_error.clear();
    if (!run || !clouds || nclouds < 1 || !out) {
        g_create_error = "dsmc_create: null argument or nclouds < 1";
        return DSMC_ERR_INVALID;
    }
    if (nclouds > KEY_MAX_CLOUDS) {
        g_create_error = "dsmc_create: at most " + std::to_string(KEY_MAX_CLOUDS) + " clouds per handle";
        return DSMC_ERR_INVALID;
    }
    *out = nullptr;
    try {
        int dev_count = 0;
        cudaError_t e = cudaGetDeviceCount(&dev_count);
        if (e != cudaSuccess || dev_count < 1) {
            g_create_error = std::string("no CUDA device: ") + cudaGetErrorString(e);
            return DSMC_ERR_CUDA;
        }
        if (run->precision == DSMC_FP32)
            *out = new Engine<float, DSMC_FP32_BLOCK, DSMC_FP32_CAP, DSMC_FP32_MINB>(*run, clouds, nclouds);
        else if (run->precision == DSMC_FP64)
            *out = new Engine<double, 256, 1536, 2>(*run, clouds, nclouds);
        else {
            g_create_error = "precision must be DSMC_FP32 or DSMC_FP64";
            return DSMC_ERR_INVALID;
        }
        return DSMC_OK;
    } catch (const Fail& f) {
        g_create_error = f.msg;
        return f.st;
    } catch (const std::exception& e) {
        g_create_error = e.what();
        return DSMC_ERR_ALLOC;
    }
}

DSMC_API dsmc_status dsmc_destroy(dsmc_handle* h) {
    delete h;
    return DSMC_OK;
}

#define NEED_H                                                                                     \
    if (!h) return DSMC_ERR_INVALID

DSMC_API dsmc_status dsmc_set_stream(dsmc_handle* h, void* s) {
    NEED_H;
    return guard(h, [&] { h->set_stream((cudaStream_t)s); });
}
DSMC_API dsmc_status dsmc_init_cloud(dsmc_handle* h, uint64_t seed) {
    NEED_H;
    return guard(h, [&] { h->init(seed); });
}
DSMC_API dsmc_status dsmc_step(dsmc_handle* h, int32_t n) {
    NEED_H;
    return guard(h, [&] { h->step(n); });
}
DSMC_API dsmc_status dsmc_batch_create(const dsmc_params* run, const dsmc_cloud_params* clouds, int32_t nclouds,
                                       dsmc_handle** out) {
    return dsmc_create(run, clouds, nclouds, out);
}
DSMC_API dsmc_status dsmc_batch_step(dsmc_handle* h, int32_t n) { return dsmc_step(h, n); }
DSMC_API dsmc_status dsmc_synchronize(dsmc_handle* h) {
    NEED_H;
    return guard(h, [&] { h->sync(); });
}
DSMC_API dsmc_status dsmc_diagnostics(dsmc_handle* h, int32_t cloud, dsmc_diag* out) {
    NEED_H;
    if (!out) return DSMC_ERR_INVALID;
    return guard(h, [&] { h->diag(cloud, out); });
}
DSMC_API dsmc_status dsmc_diagnostics_reserve(dsmc_handle* h, int32_t nslots) {
    NEED_H;
    return guard(h, [&] { h->diag_reserve(nslots); });
}
DSMC_API int64_t dsmc_diagnostics_copy_bytes(dsmc_handle* h) { return h ? h->diag_copy_bytes() : 0; }
DSMC_API dsmc_status dsmc_diagnostics_enqueue(dsmc_handle* h, int32_t slot) {
    NEED_H;
    return guard(h, [&] { h->diag_enqueue(slot); });
}
DSMC_API dsmc_status dsmc_diagnostics_collect(dsmc_handle* h, int32_t slot, int32_t cloud, dsmc_diag* out) {
    NEED_H;
    if (!out) return DSMC_ERR_INVALID;
    return guard(h, [&] { h->diag_collect(slot, cloud, out); });
}
DSMC_API dsmc_status dsmc_get_state(dsmc_handle* h, dsmc_state_buffers* out) {
    NEED_H;
    if (!out) return DSMC_ERR_INVALID;
    return guard(h, [&] { h->get_state(out); });
}
DSMC_API dsmc_status dsmc_set_state(dsmc_handle* h, const dsmc_state_buffers* in) {
    NEED_H;
    return guard(h, [&] { h->set_state(in); });
}
DSMC_API dsmc_status dsmc_get_cell_starts(dsmc_handle* h, int32_t* st, int64_t cap, int64_t* total) {
    NEED_H;
    return guard(h, [&] { h->get_cell_starts(st, cap, total); });
}
DSMC_API dsmc_status dsmc_get_sigvrmax(dsmc_handle* h, void* out, int64_t cap) {
    NEED_H;
    if (!out) return DSMC_ERR_INVALID;
    return guard(h, [&] { h->get_sigvrmax(out, cap); });
}
DSMC_API dsmc_status dsmc_set_sigvrmax(dsmc_handle* h, const void* in, int64_t n) {
    NEED_H;
    if (!in) return DSMC_ERR_INVALID;
    return guard(h, [&] { h->set_sigvrmax(in, n); });
}
DSMC_API dsmc_status dsmc_set_profiling(dsmc_handle* h, int32_t on) {
    NEED_H;
    return guard(h, [&] { h->set_profiling(on != 0); });
}
DSMC_API dsmc_status dsmc_kernel_times(dsmc_handle* h, const char** names, double* ms, int64_t* launches,
                                       int32_t cap, int32_t* count) {
    NEED_H;
    return guard(h, [&] { h->kernel_times(names, ms, launches, cap, count); });
}
DSMC_API int32_t dsmc_launches_per_step(dsmc_handle* h) { return h ? kNumStepKernels : 0; }
DSMC_API dsmc_status dsmc_check_wait_timeout(dsmc_handle* h, int32_t* bits) {
    NEED_H;
    if (!bits) return DSMC_ERR_INVALID;
    return guard(h, [&] { *bits = h->check_wait_timeout(); });
}
DSMC_API dsmc_status dsmc_adjoint_run(dsmc_handle* h, const dsmc_adj_params* p, dsmc_grad* g) {
    NEED_H;
    if (!p || !g) return DSMC_ERR_INVALID;
    return guard(h, [&] { h->adjoint_run(p, g); });
}
DSMC_API dsmc_status dsmc_adjoint_loss(dsmc_handle* h, const double* theta, double* loss, double* grad) {
    NEED_H;
    if (!loss) return DSMC_ERR_INVALID;
    return guard(h, [&] {
        double parts[2], ge[ADJ_NPARAM], gn[ADJ_NPARAM];
        h->adjoint_loss(theta, parts, grad ? ge : nullptr, grad ? gn : nullptr);
        *loss = parts[0] + parts[1];
        if (grad)
            for (int k = 0; k < ADJ_NPARAM; ++k) grad[k] = ge[k] + gn[k];
    });
}
DSMC_API dsmc_status dsmc_adjoint_loss_parts(dsmc_handle* h, const double* theta, double* parts, double* grad_energy,
                                             double* grad_retained) {
    NEED_H;
    if (!parts) return DSMC_ERR_INVALID;
    return guard(h, [&] { h->adjoint_loss(theta, parts, grad_energy, grad_retained); });
}
DSMC_API dsmc_status dsmc_set_recording(dsmc_handle* h, int32_t flags) {
    NEED_H;
    return guard(h, [&] { h->set_recording(flags); });
}
DSMC_API dsmc_status dsmc_get_evaporated(dsmc_handle* h, int32_t cloud, double* pos, double* vel, int32_t* step,
                                         int32_t* fate, int64_t cap) {
    NEED_H;
    return guard(h, [&] { h->get_evaporated(cloud, pos, vel, step, fate, cap); });
}
DSMC_API dsmc_status dsmc_get_cell_collisions(dsmc_handle* h, int32_t* counts, int64_t cap, int64_t* total) {
    NEED_H;
    return guard(h, [&] { h->get_cell_collisions(counts, cap, total); });
}
DSMC_API dsmc_status dsmc_adjoint_export_spinors(dsmc_handle* h, double* psi0, int64_t atoms_cap) {
    NEED_H;
    if (!psi0) return DSMC_ERR_INVALID;
    return guard(h, [&] { h->adjoint_export_spinors(psi0, atoms_cap); });
}
DSMC_API dsmc_status dsmc_adjoint_export(dsmc_handle* h, double* x0, double* v0, int64_t atoms_cap, int32_t* off,
                                         int64_t off_cap, int32_t* ij, double* nv, int64_t log_cap,
                                         int64_t* n_atoms, int64_t* n_log, int32_t* steps) {
    NEED_H;
    return guard(h, [&] { h->adjoint_export(x0, v0, atoms_cap, off, off_cap, ij, nv, log_cap, n_atoms, n_log, steps); });
}
DSMC_API dsmc_status dsmc_autotune(dsmc_handle* h, int32_t steps_per_candidate, int32_t* tile_atoms,
                                   double* ms_per_step) {
    NEED_H;
    return guard(h, [&] { h->autotune(steps_per_candidate, tile_atoms, ms_per_step); });
}
DSMC_API dsmc_status dsmc_autotune_table(dsmc_handle* h, int32_t* tile_atoms, int32_t* blocks_per_sm, double* ms,
                                         int32_t cap, int32_t* count, int32_t* chosen_blocks_per_sm) {
    NEED_H;
    return guard(h, [&] { h->autotune_table(tile_atoms, blocks_per_sm, ms, cap, count, chosen_blocks_per_sm); });
}

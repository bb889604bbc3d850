/*
 * dsmc.h -- C ABI of the B200 DSMC engine (libdsmc_b200.so).
 *
 * One handle simulates one or more independent atom clouds ("clouds") with the
 * Direct Simulation Monte Carlo timestep of inJeans/CUDADSMC:
 *   collide (Bird no-time-counter, s-wave) -> Larmor spin precession ->
 *   velocity-Verlet motion in the trap -> Majorana / energy-knife evaporation ->
 *   cell index -> stable sort by cell -> diagnostics.
 *
 * Conventions (all entry points):
 *   - every call returns dsmc_status (0 = DSMC_OK); dsmc_last_error() gives text;
 *   - the handle owns all device memory; callers pass host pointers only, except
 *     dsmc_set_stream (a cudaStream_t passed as void*) and the *_device calls;
 *   - all GPU work is enqueued on the handle's stream; calls on one handle are
 *     not thread-safe, separate handles are independent.
 *
 * Reference interfaces replaced (paths inside the CUDADSMC project):
 *   dsmc_create            <- cudaCalloc block + params, CUDADSMC/src/main.cu:83-140,165-174
 *   dsmc_init_cloud        <- h_initRNG + h_generateInitialDist + initSigvrmax,
 *                             CUDADSMC/src/setUp.cu:32,79,287; first index/sort main.cu:191-198
 *   dsmc_step              <- one pass of the main loop body, CUDADSMC/src/main.cu:416-523:
 *                             indexAtoms (collisions.cu:21), sortArrays (collisions.cu:275),
 *                             cellStartandEndKernel/findNumberOfAtomsInCell/exclusive_scan
 *                             (collisions.cu:228,254; main.cu:440), collide (collisions.cu:291),
 *                             evolveWavefunction (wavefunction.cu:11), moveAtoms (moveAtoms.cu:23),
 *                             evaporationTag + remove_if (evaporation.cu:68; main.cu:493),
 *                             normalise (wavefunction.cu:279)
 *   dsmc_diagnostics       <- calculateTemp (evaporation.cu:108) + atomNumber/collisionCount
 *                             snapshot fields (main.cu:526-577)
 *   dsmc_get_state/set_state <- the D2H snapshot copies, CUDADSMC/src/main.cu:526-536
 */
#ifndef DSMC_B200_H
#define DSMC_B200_H

#include <stdint.h>

#ifdef __cplusplus
#define DSMC_EXTERN extern "C"
#else
#define DSMC_EXTERN extern
#endif
#define DSMC_API DSMC_EXTERN __attribute__((visibility("default")))

#define DSMC_ABI_VERSION 2

typedef enum dsmc_status {
    DSMC_OK = 0,
    DSMC_ERR_INVALID = 1,     /* bad argument or parameter */
    DSMC_ERR_CUDA = 2,        /* CUDA runtime error (no device, launch failure...) */
    DSMC_ERR_ALLOC = 3,       /* device or host allocation failed */
    DSMC_ERR_CAPACITY = 4,    /* atom capacity exceeded */
    DSMC_ERR_CELL_FULL = 5,   /* a tile holds more atoms than it can stage (an inconsistent tiling;
                                 dense cells are split across tiles and never raise it) */
    DSMC_ERR_NAN = 6,         /* non-finite position or velocity met */
    DSMC_ERR_STATE = 7,       /* call out of order (e.g. step before init) */
    DSMC_ERR_UNSUPPORTED = 8, /* feature not available in this build / mode */
    DSMC_ERR_TIMEOUT = 9      /* a bounded device-side wait gave up */
} dsmc_status;

enum { DSMC_FP32 = 0, DSMC_FP64 = 1 };

/* Trap models. QUADRUPOLE: B = B'(x/2, y/2, -z) + B0 z^ (the linear trap of the
 * benchmark configs; B0 is an optional uniform bias).  IOFFE_PRITCHARD: the field of
 * CUDADSMC/src/moveAtoms.cu:135-142, B = B0 z^ + B'(x,-y,0) + B''/2(-xz,-yz,z^2-(x^2+y^2)/2).
 * BOX: no field, periodic boundaries on the grid box (homogeneous-gas checks). */
enum { DSMC_TRAP_QUADRUPOLE = 0, DSMC_TRAP_IOFFE_PRITCHARD = 1, DSMC_TRAP_BOX = 2 };

/* Per-cloud behaviour flags. */
enum {
    DSMC_F_COLLIDE = 1 << 0,      /* NTC collisions */
    DSMC_F_LARMOR = 1 << 1,       /* spinor precession about the local field */
    DSMC_F_MAJORANA = 1 << 2,     /* remove atoms with <sigma.B^> < 0 (evaporation.cu:90-95) */
    DSMC_F_KNIFE = 1 << 3,        /* remove atoms with E > eta(step) kB T */
    DSMC_F_NORMALISE = 1 << 4,    /* renormalise the spinor after every rotation */
    DSMC_F_KNIFE_FIXED_T = 1 << 5, /* knife uses the initial T instead of the running T */
    DSMC_F_MCWF = 1 << 6           /* spin flips and decoherence once per collision period
                                      (flipAtoms + exponentialDecay + normalise, wavefunction.cu:99-237) */
};

/* Initial distributions. */
enum {
    DSMC_INIT_THERMAL = 0, /* Boltzmann density of the trap (exact Gamma(3) sampler for the
                              quadrupole, bounded rejection sampling otherwise) */
    DSMC_INIT_UNIFORM = 1  /* uniform over the grid box (BOX trap) */
};

#define DSMC_MAX_KNOTS 9

typedef struct dsmc_cloud_params {
    int64_t n_atoms;      /* initial number of test particles */
    int64_t capacity;     /* maximum atoms (0 -> n_atoms) */
    int32_t trap;         /* DSMC_TRAP_* */
    int32_t flags;        /* DSMC_F_* */
    int32_t cells[3];     /* grid cells per axis (overflow cell added internally) */
    int32_t init_mode;    /* DSMC_INIT_* */
    double grid_min[3];   /* grid box lower corner (m) */
    double grid_max[3];   /* grid box upper corner (m) */
    double mass;          /* atom mass (kg) */
    double moment;        /* magnetic moment mu (J/T): U = mu |B|, theta = mu |B| dt / hbar */
    double B0;            /* bias field along z (T) */
    double dBdz;          /* field gradient B' (T/m) */
    double d2Bdz2;        /* field curvature B'' (T/m^2), Ioffe-Pritchard only */
    double temperature;   /* initial temperature (K) */
    double alpha;         /* real atoms per test particle */
    double sigma;         /* collision cross-section (m^2) */
    double sigvrmax_init; /* initial (sigma v_r)_max per cell (m^3/s); 0 -> sigma sqrt(16 kB T/(pi m)) */
    int32_t knife_nknots; /* piecewise-linear knife ramp eta(step), up to DSMC_MAX_KNOTS knots */
    int32_t stream_id;    /* Philox stream of this cloud (24 bits): a cloud run alone and the same
                             cloud inside a batch give identical results when their stream ids match */
    double knife_step[DSMC_MAX_KNOTS];
    double knife_eta[DSMC_MAX_KNOTS];
} dsmc_cloud_params;

typedef struct dsmc_params {
    int32_t precision;     /* DSMC_FP32 or DSMC_FP64 */
    int32_t collide_every; /* motion steps per collision step (reference: loopsPerCollision) */
    double dt;             /* timestep (s) */
    double hbar;           /* 0 -> 1.05457148e-34 (CUDADSMC/include/deviceSystemParameters.cuh:18) */
    double kB;             /* 0 -> 1.3806503e-23 */
    uint64_t seed;         /* Philox key for init (overridden by dsmc_init_cloud) and collisions */
    int32_t tile_atoms;    /* nominal atoms per tile (0 -> engine default; 128 .. tile capacity - 128).
                              Any cell occupancy is accepted: a grid cell of more atoms than a
                              tile stages beside a 512-atom tile (769 in FP32, 1025 in FP64) is
                              split across tiles and collided by its own kernel, bit for bit as
                              inside a tile. */
    int32_t use_graphs;    /* 1 -> replay captured CUDA graphs in dsmc_step (default), 0 -> plain launches */
    int32_t step_blocks_per_sm; /* blocks of the step kernel per SM (0 -> as many as fit) */
    int32_t reserved0;
} dsmc_params;

typedef struct dsmc_diag {
    int64_t step;          /* steps taken since init */
    double time;           /* simulated time (s) */
    int64_t n_alive;       /* atoms in the cloud */
    double e_kin;          /* total kinetic energy of the test particles (J) */
    double e_pot;          /* total potential energy mu |B| (J) */
    double temperature;    /* m <v^2> / (3 kB) (K) */
    double sum_v2;         /* sum of v^2 (m^2/s^2), exact fixed-point sum */
    double sum_absB;       /* sum of s |B| (T), s = +1 trapped, -1 anti-trapped: E_pot / mu; exact fixed-point sum */
    int64_t n_evaporated;  /* cumulative atoms removed (Majorana + knife) */
    int64_t n_majorana;    /* cumulative Majorana losses */
    int64_t n_knife;       /* cumulative knife losses */
    double e_evaporated;   /* cumulative energy carried away (J) */
    int64_t collisions;    /* cumulative accepted collisions */
    int64_t candidates;    /* cumulative NTC candidate pairs */
    int64_t atom_steps;    /* cumulative sum over steps of the atoms each step processed */
    int32_t error;         /* device error bits seen so far (0 = none) */
    int32_t reserved0;
} dsmc_diag;

/* Host-side view of the atom state, structure-of-arrays with 4 reals per atom
 * (float for DSMC_FP32, double for DSMC_FP64):
 *   pos[4i..4i+3] = x, y, z, atom id (integer bits in the 4th lane)
 *   vel[4i..4i+3] = vx, vy, vz, flag bits (bit 0: anti-trapped spin state)
 *   psi[4i..4i+3] = Re psi_up, Im psi_up, Re psi_dn, Im psi_dn
 * Atoms are grouped by cloud; cloud_counts[k] atoms of cloud k, in cloud order. */
typedef struct dsmc_state_buffers {
    void* pos;
    void* vel;
    void* psi;
    int64_t n;              /* in: capacity of the buffers (get) / atoms given (set); out: atoms */
    int64_t* cloud_counts;  /* nclouds entries */
} dsmc_state_buffers;

typedef struct dsmc_handle dsmc_handle;

DSMC_API int32_t dsmc_abi_version(void);
DSMC_API const char* dsmc_status_string(dsmc_status s);
DSMC_API const char* dsmc_last_error(const dsmc_handle* h);

/* Fills run and cloud parameters with one of the named workloads
 *   0: small trapped cloud, FP64 (1e4 atoms, 50^3 cells, B'=2.5 T/m, 20 uK)
 *   1: homogeneous periodic box (1e6 atoms, 100^3 cells, 10 uK, alpha = 1e4)
 *   2: full trapped step (1e7 atoms, 128^3 cells, 50 uK, Larmor + Majorana + knife 6->4)
 *   4: adjoint workload (1e6 atoms, 0.1 mT bias, 30 uK, 8-knot knife)
 * n_atoms and cells may be overridden afterwards. */
DSMC_API dsmc_status dsmc_preset(int32_t which, dsmc_params* run, dsmc_cloud_params* cloud);

DSMC_API dsmc_status dsmc_create(const dsmc_params* run, const dsmc_cloud_params* clouds,
                                 int32_t nclouds, dsmc_handle** out);
/* Batched names: many independent clouds in one handle, stepped together by one graph launch per
 * two steps.  The same calls as dsmc_create / dsmc_step (a handle always holds 1..n clouds);
 * spelled out for callers that keep batched and single-cloud code apart.  No counterpart in the
 * reference, which runs one cloud per process. */
DSMC_API dsmc_status dsmc_batch_create(const dsmc_params* run, const dsmc_cloud_params* clouds,
                                       int32_t nclouds, dsmc_handle** out);
DSMC_API dsmc_status dsmc_batch_step(dsmc_handle* h, int32_t nsteps);
DSMC_API dsmc_status dsmc_destroy(dsmc_handle* h);
DSMC_API dsmc_status dsmc_set_stream(dsmc_handle* h, void* cuda_stream);

DSMC_API dsmc_status dsmc_init_cloud(dsmc_handle* h, uint64_t seed);
DSMC_API dsmc_status dsmc_step(dsmc_handle* h, int32_t nsteps);
DSMC_API dsmc_status dsmc_synchronize(dsmc_handle* h);

/* cloud >= 0: that cloud; cloud == -1: sums over all clouds (temperature from the sums). */
DSMC_API dsmc_status dsmc_diagnostics(dsmc_handle* h, int32_t cloud, dsmc_diag* out);

/* Diagnostics read back without stopping the stream (a loop that reads every step's totals, as
 * the reference's main loop prints them, then keeps the GPU busy).  dsmc_diagnostics_reserve
 * allocates nslots slots of pinned host memory (once; a larger count reallocates, after a
 * synchronize).  dsmc_diagnostics_enqueue(h, slot) copies every cloud's step totals and the error
 * bits into that slot on the handle's stream and returns at once; dsmc_diagnostics_collect(h, slot,
 * cloud, out) waits for that copy and fills *out exactly as dsmc_diagnostics would have at the
 * enqueue (DSMC_ERR_STATE for a slot never enqueued, DSMC_ERR_INVALID outside the reserve).  A slot
 * enqueued again before it is collected holds the later copy. */
DSMC_API dsmc_status dsmc_diagnostics_reserve(dsmc_handle* h, int32_t nslots);
DSMC_API dsmc_status dsmc_diagnostics_enqueue(dsmc_handle* h, int32_t slot);
DSMC_API dsmc_status dsmc_diagnostics_collect(dsmc_handle* h, int32_t slot, int32_t cloud, dsmc_diag* out);
/* bytes one dsmc_diagnostics_enqueue copies from the device (0 for a null handle) */
DSMC_API int64_t dsmc_diagnostics_copy_bytes(dsmc_handle* h);

DSMC_API dsmc_status dsmc_get_state(dsmc_handle* h, dsmc_state_buffers* out);
DSMC_API dsmc_status dsmc_set_state(dsmc_handle* h, const dsmc_state_buffers* in);

/* Cell bookkeeping of the current sorted order: start[c] for every global cell
 * (grid cells of each cloud then its overflow cell), plus start[total] = n_alive.
 * ncells_total receives the number of global cells. */
DSMC_API dsmc_status dsmc_get_cell_starts(dsmc_handle* h, int32_t* start, int64_t capacity,
                                          int64_t* ncells_total);
/* Per-cell (sigma v_r)_max, one real per global cell (float or double). */
DSMC_API dsmc_status dsmc_get_sigvrmax(dsmc_handle* h, void* out, int64_t capacity);
DSMC_API dsmc_status dsmc_set_sigvrmax(dsmc_handle* h, const void* in, int64_t n);

/* Per-kernel device time (ms) accumulated while profiling is on; names[i] are static strings.
 * Profiling launches every kernel separately, bracketed by CUDA events on the handle's stream. */
DSMC_API dsmc_status dsmc_set_profiling(dsmc_handle* h, int32_t on);
DSMC_API dsmc_status dsmc_kernel_times(dsmc_handle* h, const char** names, double* ms,
                                       int64_t* launches, int32_t capacity, int32_t* count);
/* Number of kernel launches one dsmc_step(h, 1) issues. */
DSMC_API int32_t dsmc_launches_per_step(dsmc_handle* h);

/* Check of the bounded device-side waits (no counterpart in the reference, which has none): runs
 * the coming step's cell scan once on its own with its first scan block withheld, so that the
 * blocks after it wait for a prefix that never comes. Each gives up after about a second and sets
 * the timeout bit (64) of the device error bits, which this call writes to *bits (the scan also
 * sets 32, the bookkeeping bit, for the block left without work) and then clears. The simulation is
 * left as it was: that scan writes only what the next step's scan rewrites. Needs a handle whose
 * cells span at least two scan blocks (more than 4096 cells); takes about a second. */
DSMC_API dsmc_status dsmc_check_wait_timeout(dsmc_handle* h, int32_t* bits);

/* ---- snapshot records ------------------------------------------------------------------------
 * The reference's snapshots carry, beside the state, each atom's position and velocity at the
 * step it was tagged for loss (evapPos / evapVel by atom, zeros for atoms never lost,
 * evaporation.cu:68-106, main.cu:234-264) and each cell's accepted collisions in the last
 * collision step (collisionCount, collisions.cu:335-436, main.cu:291-304).  They cost memory and
 * stores in the step, so they are kept only when asked for.  dsmc_set_recording(h, flags) turns
 * them on (clearing them) or off; the step then writes them (no host synchronisation). */
enum {
    DSMC_REC_EVAPORATED = 1,       /* position / velocity / step / fate of every atom lost, by atom id */
    DSMC_REC_CELL_COLLISIONS = 2   /* accepted collisions of every cell in the last collision step */
};
DSMC_API dsmc_status dsmc_set_recording(dsmc_handle* h, int32_t flags);
/* Cloud `cloud`'s lost atoms by atom id (arrays of at least the cloud's capacity; NULL skips):
 * pos / vel 3 doubles each (zeros for an atom never lost), step the step it was lost in (-1:
 * never), fate how it was lost: 1 Majorana (<s.B^> < 0), 2 energy knife (0: never lost). */
DSMC_API dsmc_status dsmc_get_evaporated(dsmc_handle* h, int32_t cloud, double* pos, double* vel, int32_t* step,
                                         int32_t* fate, int64_t cap);
/* Accepted collisions per global cell (every cloud's grid cells then its overflow cell, as
 * dsmc_get_cell_starts) in the last step that ran the collisions; *total receives the cell count
 * (counts may be NULL to query it). */
DSMC_API dsmc_status dsmc_get_cell_collisions(dsmc_handle* h, int32_t* counts, int64_t cap, int64_t* total);

/* ---- pathwise adjoint ----------------------------------------------------------------------
 * Gradient of a smoothed loss of the physical run with respect to the trap gradient B', the bias
 * B0 and the knife knot heights eta_0..eta_8, with every random choice of the run held fixed.
 * dsmc_adjoint_run, called right after dsmc_init_cloud on a one-cloud quadrupole handle, runs the
 * physical simulation for `steps` steps recording every accepted collision (pair of atom ids,
 * scattering direction), then evaluates the smoothed model -- all atoms kept, spinors precessing
 * about the local field as in the run (DSMC_F_LARMOR), each atom with a survival weight multiplied
 * every step by sigmoid((cut - E)/(width kB T0)) and, when the cloud has DSMC_F_MAJORANA, by
 * sigmoid(<s.B^> / majorana_width) in place of the hard test <s.B^> < 0 -- and its adjoint through
 * Verlet, the Larmor rotation and the collision rotations, checkpointed every `checkpoint_every`
 * steps with per-segment recomputation.  Loss: L = L_E + L_N, L_E = (sum w E / sum w) / (kB T0),
 * L_N = sum w / N0; the gradient of each term is returned as well as that of their sum.
 * theta = (B', B0, eta_0 .. eta_8).  No counterpart in the reference. */
typedef struct dsmc_adj_params {
    int32_t steps;             /* physical steps recorded and differentiated */
    int32_t checkpoint_every;  /* checkpoint interval K of the smoothed model */
    int32_t precision;         /* DSMC_FP32 or DSMC_FP64 for the smoothed model and its adjoint */
    int32_t reserved0;
    double sigmoid_width_kT;   /* width of the knife's survival sigmoid in units of kB T0 */
    double majorana_width;     /* width of the Majorana survival sigmoid in <s.B^> (<= 0: 0.05) */
} dsmc_adj_params;

typedef struct dsmc_grad {
    double loss;               /* mean_energy_kT + retained_fraction */
    double mean_energy_kT;     /* L_E = sum w E / sum w / (kB T0) after the last step */
    double retained_fraction;  /* L_N = sum w / N0 */
    double dL_dBp;             /* d loss / d B' (per T/m) */
    double dL_dB0;             /* d loss / d bias (per T) */
    double dL_deta[9];         /* d loss / d knot height */
    int64_t collisions;        /* collision events recorded */
    double ms_record;          /* device time of the recorded physical run */
    double ms_forward;         /* device time of the smoothed forward pass */
    double ms_backward;        /* device time of the recomputation + adjoint pass */
    double dE_dtheta[11];      /* d L_E / d theta */
    double dN_dtheta[11];      /* d L_N / d theta */
} dsmc_grad;

DSMC_API dsmc_status dsmc_adjoint_run(dsmc_handle* h, const dsmc_adj_params* p, dsmc_grad* out);
/* Smoothed loss of the recorded run at theta (NULL: the run's own parameters); grad (11 doubles,
 * may be NULL) receives its gradient.  Same recorded collisions: central differences of this
 * function are common-random-number finite differences. */
DSMC_API dsmc_status dsmc_adjoint_loss(dsmc_handle* h, const double* theta, double* loss, double* grad);
/* The same with the two terms apart: parts[0] = L_E, parts[1] = L_N; grad_energy and
 * grad_retained (11 doubles each, may be NULL) receive their gradients. */
DSMC_API dsmc_status dsmc_adjoint_loss_parts(dsmc_handle* h, const double* theta, double* parts, double* grad_energy,
                                             double* grad_retained);
/* The recorded run's initial spinors by atom id (4 doubles each: Re u, Im u, Re d, Im d). */
DSMC_API dsmc_status dsmc_adjoint_export_spinors(dsmc_handle* h, double* psi0, int64_t atoms_cap);
/* The recorded run: initial positions and velocities by atom id (3 doubles each), per-step
 * offsets (steps + 1), collision pairs (2 ints) and directions (3 doubles).  NULL buffers skip. */
DSMC_API dsmc_status dsmc_adjoint_export(dsmc_handle* h, double* x0, double* v0, int64_t atoms_cap, int32_t* off,
                                         int64_t off_cap, int32_t* ij, double* nv, int64_t log_cap,
                                         int64_t* n_atoms, int64_t* n_log, int32_t* steps);

/* Autotuner: times dsmc_step for each candidate launch shape -- nominal tile size (atoms per
 * tile) x blocks of the step kernel per SM (how many warps walk tiles at once, which sets how much
 * of the tiles' data is in flight in L2) -- over steps_per_candidate steps and keeps the fastest;
 * the simulation advances meanwhile (results do not depend on the launch shape).  Replaces no
 * reference interface (the reference launches with cudaOccupancyMaxPotentialBlockSize or
 * 256*SMs x 512, CUDADSMC/src/main.cu:389-406). */
DSMC_API dsmc_status dsmc_autotune(dsmc_handle* h, int32_t steps_per_candidate, int32_t* tile_atoms,
                                   double* ms_per_step);
/* The last autotune's candidates and their ms per step (cap entries at most; *count receives the
 * number of candidates timed) and the chosen blocks per SM. */
DSMC_API dsmc_status dsmc_autotune_table(dsmc_handle* h, int32_t* tile_atoms, int32_t* blocks_per_sm, double* ms,
                                         int32_t cap, int32_t* count, int32_t* chosen_blocks_per_sm);

/* Sorts the n atoms of one cloud by cell without allocating any memory.  No counterpart in the
 * reference: it serves callers whose device memory is owned by another allocator (a PyTorch
 * process, for example), for whom cudaMalloc can fail on memory the pool is holding, and
 * cudaMalloc / cudaFree would synchronise the whole device.  Inputs and outputs are device
 * pointers on the current device: pos_dev holds n x 4 reals (float for DSMC_FP32, double for
 * DSMC_FP64; x, y, z used), order_dev receives n indices (order_dev[j] = input index of the atom
 * in sorted position j, stable by (cell, input index)), cell_start_dev receives
 * cells[0]*cells[1]*cells[2] + 2 ints (start of every grid cell, then of the overflow cell, then n).
 * pos_dev must be 16-byte aligned for DSMC_FP32 and 32-byte aligned for DSMC_FP64 (the positions
 * are read as vectors; DSMC_ERR_INVALID otherwise).  Work is enqueued on cuda_stream.  If a CUDA
 * error is already pending on the calling thread the call launches nothing and returns
 * DSMC_ERR_STATE, leaving that error for its owner.  Scratch lives in a fixed device array of
 * about 5.3 MB inside the library: at most 262144 atoms and 262144 grid cells per call
 * (DSMC_ERR_CAPACITY beyond).  The sort is a stable radix sort of the cell ids, so its time
 * follows the atom count whatever the cells hold.  The first call on a device (and the first
 * after a cudaDeviceReset) looks up that array's address (make it before any stream capture);
 * every call shares the array, so calls that overlap on the GPU race and must be serialised. */
DSMC_API dsmc_status dsmc_sort_cells_noalloc(const dsmc_params* run, const dsmc_cloud_params* cloud,
                                             const void* pos_dev, int64_t n, int32_t* order_dev,
                                             int32_t* cell_start_dev, void* cuda_stream);

#endif /* DSMC_B200_H */

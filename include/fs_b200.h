/* fs_b200.h -- C ABI of the B200 (sm_100a) FARRSIGHT hot path.
 *
 * Plain pointers and sizes only.  Every entry point returns an fs_status
 * (0 = FS_OK); fs_last_error() gives a message for the calling thread.
 *
 * Reference interfaces replaced (shujhan/multi_species):
 *   ElectricField::operator()(es, targets, nt, sources, q_ws, ns)
 *       inc/FieldStructure.hpp:87-93, implementations E_MQ_DirectSum
 *       src/FieldStructure.cpp:106-156 and E_MQ_Treecode :230-503
 *       -> fs_field_create / fs_field_eval / fs_field_eval_device
 *   AMRSimulation::step / rk4_step / remesh / evaluate_field(_uniform_grid)
 *       inc/AMRSimulation.hpp:113-127, src/simulation_files/AMRSimulation_step.cpp:5-263,
 *       AMRSimulation_remesh.cpp:3-48, AMRSimulation_field.cpp:5-173
 *       -> fs_sim_create / fs_sim_step / fs_sim_export
 *   AMRStructure::create_prerefined_mesh / set_leaves_weights
 *       src/structure_files/AMRStructure_amr.cpp:127-230, :1084-1151
 *       -> fs_mesh_sizes / fs_mesh_fill (host only, no GPU needed)
 */
#ifndef FS_B200_H
#define FS_B200_H

#ifdef __cplusplus
extern "C" {
#endif

typedef enum fs_status {
    FS_OK = 0,
    FS_ERR_ARG = 1,          /* invalid argument                                  */
    FS_ERR_CUDA = 2,         /* CUDA runtime error                                 */
    FS_ERR_NOMEM = 3,        /* device allocation failed / over the HBM budget     */
    FS_ERR_WALK = 4,         /* remesh point location did not converge (bounded)   */
    FS_ERR_SHIFT = 5,        /* remesh periodic shift needed > 10 shifts           */
    FS_ERR_TIMEOUT = 6,      /* a bounded device wait gave up                      */
    FS_ERR_STATE = 7,        /* call not valid in the current state                */
    FS_ERR_UNSUPPORTED = 8,  /* option not supported (e.g. open boundaries)        */
    FS_ERR_TREE = 9          /* treecode: tree deeper than the supported bound     */
} fs_status;

/* Field solver kind.  DIRECT64 is the reference arithmetic in FP64 (bit-exact
 * with E_MQ_DirectSum); DIRECT32C is the FP32 pair kernel with compensation and
 * FP64 background; TREECODE64 / TREECODE32C are the barycentric Lagrange
 * treecode of E_MQ_Treecode with an FP64 / FP32-compensated near field;
 * DIRECT64_OPEN is E_MQ_DirectSum_openbcs (src/FieldStructure.cpp:170-192),
 * open boundaries, bit-exact, field plugin only (L is ignored). */
typedef enum fs_field_kind {
    FS_FIELD_DIRECT64 = 0,
    FS_FIELD_DIRECT32C = 1,
    FS_FIELD_TREECODE64 = 2,
    FS_FIELD_TREECODE32C = 3,
    FS_FIELD_DIRECT64_OPEN = 4
} fs_field_kind;

/* Parameters of AMRSimulation::make_field_return_ptr
 * (src/simulation_files/AMRSimulation_load.cpp:49-96). */
typedef struct fs_field_params {
    double L;          /* Lx = x_max - x_min (periodic)          */
    double epsilon;    /* greens_epsilon                         */
    int kind;          /* fs_field_kind                          */
    double mac;        /* treecode MAC theta                     */
    int degree;        /* treecode interpolation degree (<= 16)  */
    int max_source;    /* treecode leaf size                     */
    int max_target;    /* accepted and ignored, as in the reference */
    int device;        /* CUDA device ordinal                    */
} fs_field_params;

typedef struct fs_field fs_field;

fs_status fs_field_create(const fs_field_params* params, fs_field** out);
fs_status fs_field_destroy(fs_field* field);

/* ElectricField::operator() drop-in (inc/FieldStructure.hpp:87-93): host
 * arrays, synchronous.  Fully overwrites es[0..nt) (undefined when the call
 * returns an error).  For the treecode kinds the
 * reference ignores targets/nt and writes es[0..ns); so does this call
 * (nt must equal ns).  Every kind is deterministic: the same inputs on the
 * same device give bit-identical es on every call. */
fs_status fs_field_eval(fs_field* field, double* es, const double* targets, int nt,
                        const double* sources, const double* q_ws, int ns);

/* Same on device pointers, enqueued on `stream` (a cudaStream_t, NULL =
 * the field's own stream); returns without synchronising. */
fs_status fs_field_eval_device(fs_field* field, double* d_es, const double* d_targets, int nt,
                               const double* d_sources, const double* d_q_ws, int ns,
                               void* stream);

/* Allocation-free self-field: E at each of n points from the same n points
 * (targets == sources, the simulation's use), FP32-compensated like
 * FS_FIELD_DIRECT32C, on device pointers, synchronous on `stream` (a
 * cudaStream_t, NULL = the legacy default stream).
 * No counterpart in the reference: it exists for callers that cannot allocate
 * device memory at call time (a pool or arena that owns the device, hosts that
 * allocate only at start-up, threads where cudaMalloc's device-wide
 * synchronisation is not allowed).  All scratch lives in one static device
 * array of about 9.5 MiB that each GPU loading the library keeps until exit;
 * n is limited to 32768 (larger n returns FS_ERR_ARG).  The first call on a
 * device looks up the array's device address (cudaGetSymbolAddress) for that
 * device.  The call waits for its own work: it returns after d_es is written
 * (or the error is known).  Calls share the
 * array, so calls that overlap on one GPU race: serialise them.  The looked-up
 * address is kept for the life of the process; after cudaDeviceReset on a
 * device, reload the library before calling this again there.  When the call
 * returns an error, d_es[0..n) is undefined. */
fs_status fs_field_eval_noalloc(double L, double epsilon, double* d_es, const double* d_x,
                                const double* d_q_ws, int n, void* stream);

/* Test hook for the failure paths (no counterpart in the reference): the
 * bounds of the library's device waits on `device`.  mbar_polls is how many
 * times a pair kernel polls for a source tile before it reports
 * FS_ERR_TIMEOUT (0 = give up at once; < 0 = the default bound); walk_panels is
 * how many panels a remesh point-location walk may visit before it reports
 * FS_ERR_WALK (<= 0 = the default, 1024).  The bounds are per device and apply
 * to every later launch until changed.  A call that fails this way leaves its
 * outputs undefined; the field object or session itself stays usable (a failed
 * remesh leaves the state it started from). */
fs_status fs_debug_set_wait_limits(int device, long long mbar_polls, int walk_panels);

/* ------------------------------------------------------------------ session */
/* One species of the deck (AMRSimulation_load.cpp:188-270 keys). */
typedef struct fs_species_params {
    double q, m;
    int initial_height, p_height;
    double pmin, pmax;
    int ics_type;                 /* 1,2 Landau; 3 strong two-stream; 4 colder two-stream;
                                     5 Friedman beam; 6 Maxwell-Juttner; 7 relativistic
                                     two-stream; 8 relativistic travelling wave; 9,10 ion
                                     acoustic (make_f0_return_ptr,
                                     AMRSimulation_load.cpp:139-225)                    */
    double pth, pstr, amp, normalized_wavenumber;
    /* Adaptive refinement (AMRSimulation_load.cpp:246-258; generate_mesh,
     * AMRStructure_amr.cpp:901-941): when on, panels of the uniform mesh whose
     * nine f values meet a criterion of amr_eps (spread, relative spread,
     * max/min, x and p difference quotients, in that order) are split 2x2 up to
     * max_height, at the start and at every remesh. */
    int do_adaptively_refine;
    int max_height;
    int n_amr_eps;                /* 0..5; 0 turns the refinement off           */
    double amr_eps[5];
    /* Deck keys of the relativistic initial conditions: "mu" (inverse
     * temperature of ics 6 and 7; the reference's default 1.0 when the key is
     * absent) and "wave_beta" (ics 8; default 0.8). */
    double mu;
    double wave_beta;
} fs_species_params;

/* Deck-level parameters (AMRSimulation_load.cpp:14-47). */
typedef struct fs_sim_params {
    double xmin, xmax;
    int quadrature;               /* 0 trapezoid, 1 Simpson                     */
    double dt;
    int remesh_period;
    double greens_epsilon;
    int field_kind;               /* fs_field_kind                              */
    double mac;
    int degree;
    int max_source;
    int num_species;              /* 1..8                                       */
    fs_species_params species[8];
    int device;
    /* Drive field added to E at every evaluation, at the evaluation's time
     * (deck "external_field", AMRSimulation_load.cpp:98-136; ExternalTanh /
     * ExternalSine / ExternalLogistic, src/FieldStructure.cpp:15-96). */
    int use_external_field;       /* 0 off                                      */
    int external_type;            /* 0 tanh, 1 sine, 2 logistic                 */
    double external_Am, external_k, external_omega;
    /* Opt-in relativistic position push: every RK4 stage moves x with
     * v = (p/m) / sqrt(1 + (p/m)^2) instead of p (the formula of
     * AMRSimulation::relativistic_momentum_push, AMRSimulation_step.cpp:101-111).
     * The reference defines that push but never calls it, and its
     * "relativistic" deck key has no effect on rk4_step; 0 keeps that
     * behaviour. */
    int relativistic_push;
} fs_sim_params;

typedef struct fs_sim fs_sim;

/* AMRSimulation ctor (src/simulation_files/AMRSimulation.cpp:5-91): builds the
 * meshes on the host, f0 and weights, uploads the state and evaluates the
 * initial reduced-grid field on the device. */
fs_status fs_sim_create(const fs_sim_params* params, fs_sim** out);
fs_status fs_sim_destroy(fs_sim* sim);
/* nsteps x AMRSimulation::step (AMRSimulation_step.cpp:5-99), device resident,
 * synchronous on return. */
fs_status fs_sim_step(fs_sim* sim, int nsteps);
/* AMRSimulation::remesh (AMRSimulation_remesh.cpp:3-48) on the current state:
 * every species is interpolated onto its fresh mesh and the reduced-grid field
 * is evaluated.  fs_sim_step calls it every remesh_period steps. */
fs_status fs_sim_remesh(fs_sim* sim);
/* Total points (species = -1) or the points of one species. */
fs_status fs_sim_num_points(const fs_sim* sim, int species, int* n);
/* Copy the concatenated state (species in deck order) to host arrays; any
 * pointer may be NULL (AMRSimulation::scatter / write_to_file). */
fs_status fs_sim_export(fs_sim* sim, double* xs, double* ps, double* fs, double* q_ws, double* es);
/* Overwrite positions/velocities of the current state from host arrays (for
 * tests that inject a given state; weights and f are kept). */
fs_status fs_sim_import_xp(fs_sim* sim, const double* xs, const double* ps, const double* es);
fs_status fs_sim_iter(const fs_sim* sim, int* iter, double* t);
/* Pair interactions evaluated so far (full + reduced), for throughput metrics. */
fs_status fs_sim_pair_count(const fs_sim* sim, double* pairs);
/* Direct-equivalent pairs (N^2 per evaluation) and kernel-level evaluations
 * (treecode: near pairs + far cluster terms; counted while profiling is
 * enabled, otherwise equal to the direct-equivalent count). */
fs_status fs_sim_work(const fs_sim* sim, double* direct_pairs, double* kernel_evals);

/* The initial distribution of species `species` of a deck at n phase-space
 * points (distribution::operator() of the object make_f0_return_ptr builds,
 * AMRSimulation_load.cpp:139-225, initial_distributions.cpp:11-460).  Host
 * only: no device is touched.  Points where the reference would read past its
 * tabulated Friedman-beam density or travelling-wave orbit are rejected with
 * FS_ERR_ARG instead. */
fs_status fs_initial_f0(const fs_sim_params* params, int species, int n, const double* x,
                        const double* p, double* f);

/* ------------------------------------------------------------------ batch */
/* Many independent simulations stepped together on one device and stream
 * (no counterpart in the reference, which runs one deck per process).  Each
 * of a step's four field evaluations runs every member's preparation, then
 * the FP32 pair work of all FS_FIELD_DIRECT32C members as one persistent
 * launch over work items taken longest first; other kinds evaluate on their
 * own in the same stream.  Results equal those of fs_sim_step on each member
 * alone (the pair sums are made in the same fixed order).  The first step
 * times the candidate item shapes and keeps the fastest; later steps of
 * all-direct batches are captured once per remesh pattern into a CUDA graph
 * and replayed.  Adding or removing a member discards the graphs. */
typedef struct fs_batch fs_batch;

fs_status fs_batch_create(int device, fs_batch** out);
fs_status fs_batch_destroy(fs_batch* batch);
/* Create a member (as fs_sim_create; params->device must be the batch's). */
fs_status fs_batch_add(fs_batch* batch, const fs_sim_params* params, int* id);
fs_status fs_batch_remove(fs_batch* batch, int id);
/* nsteps steps of every member, synchronous on return. */
fs_status fs_batch_step(fs_batch* batch, int nsteps);
/* As fs_sim_export for member `id`. */
fs_status fs_batch_export(fs_batch* batch, int id, double* xs, double* ps, double* fs, double* q_ws, double* es);
/* Points, steps taken, time and pair interactions of member `id` (NULL to skip). */
fs_status fs_batch_info(fs_batch* batch, int id, int* npoints, int* iter, double* t, double* pairs);
/* Device time of each step of the last fs_batch_step call, ms. */
fs_status fs_batch_step_times(fs_batch* batch, double* ms, int cap, int* n);
/* Pair interactions of all members so far. */
fs_status fs_batch_work(fs_batch* batch, double* pairs);
/* Chosen item shape (targets per thread, source tiles of 256 per item) and
 * the number of steps replayed from graphs / run launch by launch. */
fs_status fs_batch_stats(fs_batch* batch, int* targets_per_thread, int* tiles_per_item, long long* graph_steps,
                         long long* plain_steps);
/* For the FP32-compensated members' last field evaluation (no counterpart in
 * the reference): the pairs evaluated in FP64 (|d| <= 16 epsilon) and all
 * pairs, so that a caller can bound the pair kernel by the FP32 pipe for the
 * far pairs and the FP64 pipe for the band pairs.  Synchronises the batch. */
fs_status fs_batch_band_pairs(fs_batch* batch, double* band_pairs, double* pairs);
/* Fix the item shape instead of autotuning (targets per thread 4 or 8, source
 * tiles per item >= 1).  Pair sums are then made in the same order whatever
 * the other members are, so a member's results are bit-identical alone and in
 * any mix. */
fs_status fs_batch_set_tuning(fs_batch* batch, int targets_per_thread, int tiles_per_item);
/* Graph capture on (default) or off; either way discards existing graphs. */
fs_status fs_batch_set_graphs(fs_batch* batch, int on);

/* ------------------------------------------------------------------ pool */
/* Request loop for serving many simulations on one device (no counterpart in
 * the reference).  Client threads submit (deck, steps) requests and return at
 * once; one device-owner thread admits queued requests in arrival order while
 * the estimated device bytes of the live members stay within
 * hbm_budget_bytes and fewer than max_live are running, steps every live
 * member together (an fs_batch underneath: their FP32 pair work shares one
 * launch per field evaluation), and retires finished members (final state to
 * host memory, device state freed).  Requests arriving while others run join
 * at the next step.  All fs_pool_* calls are thread-safe. */
typedef struct fs_pool_params {
    int device;
    double hbm_budget_bytes;      /* e.g. 150e9                                        */
    int max_live;                 /* running requests at most (slots)                  */
    int targets_per_thread;       /* 0: autotune on the first step; else 4 or 8        */
    int tiles_per_item;           /* with targets_per_thread != 0: source tiles per item */
} fs_pool_params;

typedef enum fs_request_state {
    FS_REQ_QUEUED = 0,
    FS_REQ_RUNNING = 1,
    FS_REQ_DONE = 2,
    FS_REQ_FAILED = 3,
    FS_REQ_CANCELLED = 4
} fs_request_state;

typedef struct fs_request_info {
    int state;                    /* fs_request_state                                  */
    int steps_done, nsteps, npoints;
    double pairs;                 /* pair interactions evaluated for it                */
    double step_ms_p50, step_ms_p99;  /* its per-step latencies (wall time of the steps it took part in) */
    double queue_ms;              /* submit -> admission (-1 while queued)             */
    double total_ms;              /* submit -> completion (-1 until finished)          */
    char error[256];
} fs_request_info;

typedef struct fs_pool_stats_t {
    long long submitted, admitted, completed, failed, cancelled, queued, live, iterations;
    double hbm_in_use_bytes;      /* estimated bytes of the live members               */
    double pairs;                 /* pair interactions of all requests                 */
    double busy_ms;               /* wall time spent stepping                          */
    double step_ms_p50, step_ms_p99;  /* over every (request, step)                    */
} fs_pool_stats_t;

typedef struct fs_pool fs_pool;

fs_status fs_pool_create(const fs_pool_params* params, fs_pool** out);
/* Stops the loop: queued and running requests are cancelled. */
fs_status fs_pool_destroy(fs_pool* pool);
/* Queue a simulation of params for nsteps steps.  FS_ERR_NOMEM when its
 * estimate alone exceeds the budget. */
fs_status fs_pool_submit(fs_pool* pool, const fs_sim_params* params, int nsteps, long long* id);
fs_status fs_pool_cancel(fs_pool* pool, long long id);
fs_status fs_pool_poll(fs_pool* pool, long long id, fs_request_info* info);
/* Block until the request finished (timeout_ms < 0: no limit); *state gets its state. */
fs_status fs_pool_wait(fs_pool* pool, long long id, double timeout_ms, int* state);
/* Final state of a completed request (as fs_sim_export; any pointer may be NULL). */
fs_status fs_pool_result(fs_pool* pool, long long id, double* xs, double* ps, double* fs, double* q_ws, double* es);
/* Forget a finished request and its host copy of the state. */
fs_status fs_pool_release(fs_pool* pool, long long id);
fs_status fs_pool_step_times(fs_pool* pool, long long id, double* ms, int cap, int* n);
fs_status fs_pool_stats(fs_pool* pool, fs_pool_stats_t* stats);
/* Device bytes the pool reserves for a simulation of these parameters. */
fs_status fs_pool_estimate_bytes(const fs_sim_params* params, double* bytes);

/* ----------------------------------------------------- diagnostic output */
/* Write the reference's diagnostic and restart files for this session
 * (AMRStructure::write_to_file, AMRStructure_io.cpp:8-101 and
 * AMRStructure_restart.cpp:33-98; evaluate_field_uniform_grid's reduced-grid
 * dump, AMRSimulation_field.cpp:81-111) under <sim_dir>simulation_output/:
 * <species>/{xs/xs_,ps/ps_,fs/fs_}<iter> (raw FP64),
 * <species>/panels/leaf_point_inds_<iter> (int32 x 9 per leaf),
 * <species>/panels/full_tree_<iter> (int64 count + 80-byte panel records),
 * reduce_xs/xs_<iter> and reduced_es/es_<iter> (raw FP64).  Particle files are
 * written now (the constructor's dump) and after every step whose iteration is a
 * multiple of diag_phase_space_period; reduced-grid files at reduced
 * evaluations (start, remesh) on multiples of diag_period.  Copies go to pinned
 * host memory on the session's stream and a writer thread writes the files
 * while the next steps run.  species_names (num_species entries, NULL = species0,
 * species1, ...) name the directories.  Directories are created as needed. */
fs_status fs_sim_set_output(fs_sim* sim, const char* sim_dir, const char* const* species_names, int diag_period,
                            int diag_phase_space_period);
/* Restart from the files of iteration `iter` under <sim_dir>simulation_output/
 * (the reference's restart, AMRSimulation.cpp:65-84 and AMRStructure_restart.cpp:
 * 101-229): per species xs/ps/fs and full_tree; weights from the loaded leaves
 * at the loaded positions, as the reference computes them (so a restart
 * continues a run exactly from a dump taken right after a remesh),
 * t = iter * dt, then the reduced-grid field on the loaded state.  The session
 * must come from the same deck (a uniform species must load its mesh's point
 * count).  Missing or malformed files return FS_ERR_ARG and leave the session
 * as it was. */
fs_status fs_sim_restart(fs_sim* sim, const char* sim_dir, const char* const* species_names, int iter);
/* Wait until every queued file is written; FS_ERR_STATE if a write failed. */
fs_status fs_sim_flush_output(fs_sim* sim);

/* ------------------------------------------------------------- host mesh */
/* Sizes of the uniform periodic panel mesh of create_prerefined_mesh. */
fs_status fs_mesh_sizes(int initial_height, int p_height, int* npoints, int* npanels, int* nleaves);
/* Fill points (reference point order), panels (18 ints each: point_inds[9],
 * level, parent, which_child, child_start, left, top, right, bottom, flags
 * 1 left-bdry 2 right-bdry 4 refined-xp 8 refined-p), leaves (DFS order) and
 * base quadrature weights q*dx*dp*stencil (before the *f of set_leaves_weights).
 * Any output pointer may be NULL. */
fs_status fs_mesh_fill(int initial_height, int p_height, double xmin, double xmax, double pmin,
                       double pmax, double q, int quadrature, double* xs, double* ps, int* panels,
                       int* leaves, double* base_weights);

/* Device time of each step of the last fs_sim_step call, in ms, measured with
 * CUDA events on the simulation's stream; *n receives the count (<= cap). */
fs_status fs_sim_step_times(const fs_sim* sim, double* ms, int cap, int* n);

/* ------------------------------------------------------------- profiling */
/* When enabled, the library brackets its dominant kernels (pair kernels,
 * treecode near/far kernels, remesh kernels) with CUDA events on the stream
 * they are launched on.  fs_profile_read synchronises on the pending events and
 * returns the launches, summed device time and summed algorithmic work (pair
 * interactions for field kernels) of kernels named `kernel` (e.g.
 * "k_pairs32", "k_direct64", "remesh"). */
fs_status fs_profile_enable(int on);
fs_status fs_profile_read(const char* kernel, long long* launches, double* total_ms, double* total_work);
fs_status fs_profile_reset(void);

/* ------------------------------------------------------------- misc */
const char* fs_last_error(void);
int fs_version(void);
/* Kernels launched by this library in this process so far. */
long long fs_kernel_launches(void);

#ifdef __cplusplus
}
#endif
#endif /* FS_B200_H */

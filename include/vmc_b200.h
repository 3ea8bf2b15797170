/* vmc_b200.h — C ABI of the B200 walker engine (vmachine_b200/libvmc_b200.so).
 *
 * Plain C types only: pointers and sizes, no torch or CUDA types in a signature.
 * Conventions:
 *   - return 0 on success, a negative VMC_E_* code on failure (never exits);
 *   - host pointers belong to the caller and are copied in or out;
 *   - calls on one engine are stream-ordered and not re-entrant; separate
 *     engines may be driven from separate host threads;
 *   - matrices are row-major; a parameter matrix is n_elements x p_max, rows in
 *     the configuration's element order, as the reference's m_parameters
 *     (src/system.h:335).
 *
 * Each entry point names the reference (evenmn/VMaChine) interface it replaces.
 */
#ifndef VMC_B200_H
#define VMC_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define VMC_ABI_VERSION 6

enum {
    VMC_OK = 0,
    VMC_E_CONFIG = -1,      /* input.in error: unknown key, bad value (parser.cpp:314-320 aborts) */
    VMC_E_UNSUPPORTED = -2, /* a configuration the engine does not implement                   */
    VMC_E_CUDA = -3,        /* CUDA runtime error                                              */
    VMC_E_ARG = -4,         /* bad argument (size, NULL)                                       */
    VMC_E_NAN = -5,         /* NaN kinetic energy (sampler.cpp:219-225 aborts with 143), or a NaN
                               energy average: no optimiser step is taken                     */
    VMC_E_SINGULAR = -6,    /* singular Slater block at (re)initialisation                     */
    VMC_E_STATE = -7,       /* call out of order (e.g. sampling before walkers exist)          */
    VMC_E_TIMEOUT = -8,     /* a bounded device wait gave up: the pass is incomplete, its sums
                               are not applied; vmc_init_walkers or vmc_load_state clears it  */
};

enum { VMC_PRECISION_FP64 = 0, VMC_PRECISION_MIXED = 1 };

typedef struct vmc_engine vmc_engine;

typedef struct {
    int device;            /* CUDA device ordinal (default 0)                         */
    int precision;         /* VMC_PRECISION_*; overrides the `precision:` key if >= 0  */
    int num_walkers;       /* overrides `numWalkers:` if > 0                           */
    int walkers_per_block; /* CTA shape override if > 0 (else autotuned)               */
    int refresh_interval;  /* FP64 rebuild cadence in steps (mixed); <0 = config/auto  */
    int compat;            /* 1 = reproduce reference quirks, 0 = corrected, <0 = config */
} vmc_options;

/* Read-only description of an engine (System getters, src/system.h:171-200). */
typedef struct {
    int n_particles, n_dimensions, n_coords;    /* N, d, D = N d                       */
    int n_elements, p_max;                      /* parameter matrix shape              */
    int n_walkers, precision, sampling;         /* sampling: 0 importance, 1 brute force */
    int steps_per_walker, burn_in, batches;     /* per-iteration schedule              */
    int n_iterations, compat;
    int n_accumulators;                         /* per walker: 9 + 2 x accumulated parameters */
    int walkers_per_block, refresh_interval;
    int element_kind[8];                        /* VMC_ELEM_* in configuration order    */
    int kernel_variant;                         /* VMC_KERNEL_* of the sweep            */
    int walkers_per_warp;                       /* production sweep: 1, or 2 (small dots) */
    int sweep_form;                             /* VMC_SWEEP_* of the production sweep    */
} vmc_info;

/* Forms of the production sweep: the walker record staged in shared memory (one, two
 * or four walkers per warp), or the dots' owner form (one walker per warp, each lane
 * holding two particles' state in registers; `sweepForm:` key). */
enum { VMC_SWEEP_STAGED = 1, VMC_SWEEP_OWNER = 2 };

/* Sweep implementations: element flags read at run time, the quantum-dot flag
 * set compiled in, or the general FP64 path (SimpleJastrow, RBM, hydrogen orbitals). */
enum { VMC_KERNEL_RUNTIME_FLAGS = 0, VMC_KERNEL_DOT = 1, VMC_KERNEL_GENERAL = 2 };

enum {
    VMC_ELEM_GAUSSIAN = 0,
    VMC_ELEM_SLATER = 1,
    VMC_ELEM_PADE = 2,
    VMC_ELEM_SIMPLEJASTROW = 3,
    VMC_ELEM_RBMGAUSSIAN = 4,
    VMC_ELEM_RBMPRODUCT = 5,
    VMC_ELEM_HYDROGENLIKE = 6,
};

/* Per-iteration totals over all walkers (the reduced form of the Sampler's
 * cumulative members, sampler.cpp:111-187), compensated FP64. */
typedef struct {
    double energy, energy2, kinetic, kinetic2, external, external2, interaction, interaction2;
    double accepts;
    double n_samples;     /* sampled steps summed over walkers                       */
    double n_window;      /* gradient-window normaliser: walkers x steps-per-batch     */
    double seconds;       /* device time of the iteration's kernels                  */
    double sweep_seconds; /* device time of the sweep kernel launches alone            */
    double sweep_launches;/* number of sweep kernel launches                           */
    double max_drift;     /* mixed precision: largest |inverse - FP64 rebuild| / |inverse| seen */
    double q99_drift;     /* its 99th percentile over walkers (drives refreshInterval: auto) */
    uint32_t status;      /* OR of walker status bits (1 NaN energy, 2 bad ratio, 4 singular) */
} vmc_sums;

/* Averages after an iteration (Sampler::computeAverages, sampler.cpp:194-226). */
typedef struct {
    double energy, std_error, kinetic, external, interaction, acceptance;
    double walker_std_error; /* std of per-walker means / sqrt(W): independent chains */
} vmc_averages;

/* Version of this ABI, for a binding to check (no counterpart in the reference). */
int vmc_abi_version(void);

/* Parse input.in text and build an engine on a device.  Replaces
 * System::parser + System::initializeSystem (parser.cpp:25-333, system.cpp:50-73).
 * `opt` may be NULL.  Walkers are created by vmc_init_walkers. */
int vmc_create(const char *input_in_text, const vmc_options *opt, vmc_engine **out);
/* Frees the engine and its device memory (System::~System, system.cpp:231). */
void vmc_destroy(vmc_engine *e);
/* Sizes and choices of the engine (System's getters, system.h:171-181, plus the
 * engine's own: walkers, precision, kernel form). */
int vmc_get_info(const vmc_engine *e, vmc_info *out);
/* Last error message (static storage, for the calling thread's last failure). */
const char *vmc_last_error(void);

/* Parameter matrix in/out (System::updateAllParameters, elementoperation.cpp:68-73). */
int vmc_set_parameters(vmc_engine *e, const double *theta, int n_elements, int p_max);
int vmc_get_parameters(const vmc_engine *e, double *theta, int n_elements, int p_max);

/* Walker start: pos = W x D coordinates (particle-major, k = p d + dim), or NULL for
 * the configured InitialState from per-walker Philox(seed) streams
 * (randomnormal.cpp:10-25 / randomuniform.cpp:10-24), then the element arrays
 * (WaveFunction::initializeArrays) and the importance-sampling force cache
 * (ImportanceSampling::initialize, importancesampling.cpp:11-32). */
int vmc_init_walkers(vmc_engine *e, const double *pos, uint64_t seed);
/* Every walker's positions (System::getPositions, system.h:212). */
int vmc_get_positions(const vmc_engine *e, double *pos /* W x D */);

/* One sampling pass of every walker: `burn_in` unsampled then sampled steps,
 * `steps` in all (System::runMetropolisCycles, system.cpp:147-164, with
 * Metropolis::acceptMove and Sampler::sample).  `iteration` selects the gradient
 * window (sampler.cpp:82-86).  Totals are reduced on the device. */
int vmc_sample(vmc_engine *e, int iteration, int steps, int burn_in, vmc_sums *out,
               double *grad_sum /* n_elements x p_max */,
               double *egrad_sum /* n_elements x p_max */);

/* One optimisation iteration (System::runSimulation body, system.cpp:93-138):
 * vmc_sample with the configured schedule, averages, optimiser step
 * (ADAM/SGD/GD, optimization.cpp:10-16, adam.cpp:22-37, sgd.cpp:23-28,
 * gradientdescent.cpp:24-29), parameter update.  Returns the averages. */
int vmc_run_iteration(vmc_engine *e, int iteration, vmc_averages *out);

/* The host half of an iteration, from totals that may be summed over several
 * engines (one per GPU): averages (Sampler::computeAverages, sampler.cpp:194-226),
 * the optimiser step and the parameter update (system.cpp:110-137).  Every engine
 * that applies the same totals ends with the same parameters, which is what the
 * reference's MPI_Reduce + MPI_Bcast achieve (sampler.cpp:111-187,
 * system.cpp:130-135).  vmc_run_iteration = vmc_sample + vmc_apply_sums. */
int vmc_apply_sums(vmc_engine *e, const vmc_sums *total, const double *grad_sum,
                   const double *egrad_sum, vmc_averages *out);

/* Per-walker sampled-energy means of the last vmc_sample (W values): each walker's
 * m_cumulativeEnergy / steps, what one reference rank holds before the MPI_Reduce
 * (sampler.cpp:111-187). */
int vmc_get_walker_energies(const vmc_engine *e, double *mean_energy);

/* Oracle entry (a): evaluate every walker at its current positions after an FP64
 * rebuild: per element gradient (W x E x D), Laplacian (W x E), parameter
 * gradient (W x E x p_max), and {T, V_ext, V_int} (W x 3).  Replaces
 * WaveFunction::computeGradient/computeLaplacian/computeParameterGradient plus
 * System::getKineticEnergy, Hamiltonian::getExternalEnergy and
 * Interaction::getInteractionEnergy (elementoperation.cpp:95-123). */
int vmc_eval(vmc_engine *e, double *grad, double *lap, double *pgrad, double *energies);

/* Move coordinate k[w] of walker w to xnew[w] through the incremental update path
 * (System::updateAllArrays + evaluateRatio, elementoperation.cpp:38-47,80-87) and
 * keep it; per element |Psi|^2 ratios go to ratios (W x E). */
int vmc_probe_move(vmc_engine *e, const int *k, const double *xnew, double *ratios);

/* Oracle entry (b): run `steps` Metropolis steps consuming a caller stream of
 * W x steps x 3 doubles {u_k, z (importance) or u (brute force), u_accept} in
 * place of the RNG (RandomNumberGenerator::nextInt/nextGaussian/nextDouble,
 * rng.h:6-22).  Records accept flags (W x steps) and {T, V_ext, V_int} per step
 * (W x steps x 3); either may be NULL.  stream == NULL records a run on the
 * engine's own per-walker Philox streams instead. */
int vmc_replay(vmc_engine *e, const double *stream, int steps, uint8_t *accepted,
               double *energies);

/* Replace the RNG of subsequent vmc_sample / vmc_run_iteration calls by a caller
 * stream of W x length x 3 doubles (same layout as vmc_replay), consumed in order
 * across calls; NULL restores the Philox streams.  Lets a whole iteration be
 * replayed against the reference's ReplayRNG-driven run. */
int vmc_set_replay(vmc_engine *e, const double *stream, int length);

/* Per-walker status words (OR of VMC status bits) since creation (no counterpart in
 * the reference, which aborts or carries on instead). */
int vmc_get_status(const vmc_engine *e, uint32_t *status /* W */);

/* Full run as System::runSimulation (system.cpp:81-139) without terminal output:
 * iterations until the last one (numIterations, or rangeOfAdaptiveSteps + 1 after
 * convergence with checkConvergence: tolerance / numberOfEnergies), with
 * applyAdaptiveSteps' longer last iterations (additionalSteps,
 * additionalStepsLastIter), weights_<it>.dat every checkpointFreq iterations
 * (printParametersToFile), energy.dat / kinetic.dat / external.dat / interaction.dat
 * (printEnergyToFile), and in the last iteration the densities (onebody.dat,
 * onebody2.dat, twobody.dat; computeOneBodyDensity / 2, computeTwoBodyDensity,
 * numberOfBins, maxRadius) and the blocking of its energies (doResampling; see
 * vmc_last_blocking), files in `path`.  Per-iteration averages to `history` (may be
 * NULL, n_history entries).  Returns the number of iterations run (>= 0) or a
 * negative error. */
int vmc_run_simulation(vmc_engine *e, vmc_averages *history, int n_history);

/* Device-side stopwatch on the engine's stream: mode 0 records the start; mode 1
 * records the stop, waits for it and writes the elapsed milliseconds (the
 * reference times each iteration with MPI_Wtime, system.cpp:101-104). */
int vmc_stopwatch(vmc_engine *e, int mode, double *ms);

/* FP64 rebuild cadence of a mixed-precision engine, in steps (>= 1): engines that
 * share one population (walker shards on several GPUs) set the same cadence after
 * each iteration, so every shard refreshes where one engine over all walkers would;
 * with `refreshInterval: auto` the drift test goes on tuning from this value.  No
 * counterpart in the reference (which never re-inverts). */
int vmc_set_refresh_interval(vmc_engine *e, int steps);

/* FMA throughput of a device, FP32 (VMC_PRECISION_MIXED) or FP64, measured with a
 * register-resident loop over all SMs; TFLOP/s counting an FMA as 2 flops.  The
 * roofline denominator of the CUDA-core-bound sweep kernel (no counterpart in the
 * reference). */
int vmc_measure_fma_peak(int device, int precision, double *tflops);

/* ---- Blocking analysis (Sampler::doResampling, sampler.cpp:319-405, and the
 * Blocker of include/block/blocker.cpp:10-71: automatic blocking, M. Jonsson,
 * Phys. Rev. E 98, 043304 (2018)) ---- */
typedef struct {
    double mean;          /* Blocker::mean                                            */
    double std_error;     /* Blocker::stdErr = sqrt(mse_mean)                         */
    double mse_mean;      /* Blocker::mse_mean: variance of the mean at the chosen level */
    double mse_std_error; /* Blocker::mse_stdErr = (2 nK - 1) mse_mean^2 / nK^2        */
    long long n_k;        /* Blocker::nK: blocks at the chosen level                  */
} vmc_block;

typedef struct {
    /* the walkers' series concatenated walker by walker (the reference's instant
     * files appended over ranks, walkers in place of ranks); every field -1 unless
     * n_walkers x samples_per_walker is a power of two (blocker.cpp:20-25) */
    vmc_block energy, kinetic, external, interaction;
    /* independent chains: mean of the walkers' means; mse_mean = sum over walkers of
     * each walker's own blocked variance of its mean / W^2 (n_k = 0) */
    vmc_block energy_walkers;
    long long samples_per_walker; /* 2^d: the first 2^d sampled steps of each walker */
} vmc_blocking_result;

/* Blocker on a host series of n values; n not a power of two: every field -1 and
 * n_k = 0 (the reference prints an error and sets -1). */
int vmc_block_series(const double *x, long long n, vmc_block *out);
/* `steps` moves per walker with the current parameters (no optimiser step; sums as
 * vmc_sample with iteration 0), recording every walker's (T, V_ext, V_int) per step
 * in device memory (W x steps x 24 bytes, released after), then blocking of E_L, T,
 * V_ext and V_int on the device.  Consumes a replay stream set by vmc_set_replay. */
int vmc_blocking(vmc_engine *e, int steps, int burn_in, vmc_blocking_result *out);
/* The blocking of the last iteration of the latest vmc_run_simulation with
 * doResampling: true (Sampler::doResampling; the record must fit in 16 GB of device
 * memory, W x steps x 24 bytes, else there is none: VMC_E_STATE). */
int vmc_last_blocking(const vmc_engine *e, vmc_blocking_result *out);

/* ---- Electron densities (Sampler::computeOneBodyDensity, computeOneBodyDensity2,
 * computeTwoBodyDensity, sampler.cpp:639-692) ----
 * `steps` moves per walker with the current parameters (no optimiser step; sums as
 * vmc_sample with iteration 0), counting every sampled step of every walker into the
 * requested histograms (NULL: not computed), bins = numberOfBins, step = max_radius /
 * bins: radial[bins] counts floor(r / step) for r < max_radius; spatial[bins][bins]
 * counts the cell (trunc(y / 2 step) + bins/2, trunc(x / 2 step) + bins/2) inside the
 * grid (row = y); two_body[bins][bins] counts (floor(r_i / step) + 1, floor(r_j / step)
 * + 1) for pairs i < j with both below bins.  64-bit counts summed over walkers. */
int vmc_densities(vmc_engine *e, int steps, int burn_in, int bins, double max_radius, uint64_t *radial,
                  uint64_t *spatial, uint64_t *two_body);

/* ---- Checkpoint and resume ----
 *
 * Parameter files in the reference's text format (Sampler::printParametersToFile,
 * sampler.cpp:507-515, read by FromFile, fromfile.cpp:30-79): one row per element,
 * Eigen's default layout (common right-aligned width, one space between values).
 * digits <= 0: 6 significant digits, the reference's files byte for byte; 17 keeps
 * every bit.  vmc_run_simulation writes <path>weights_<it>.dat every checkpointFreq
 * iterations when printParametersToFile is true (system.cpp:116-118). */
/* The text of a parameter file for an n_elements x p_max matrix into buf (at most
 * cap - 1 characters and a zero); returns its full length, or < 0 on error. */
long long vmc_format_weights(const double *theta, int n_elements, int p_max, int digits, char *buf,
                             long long cap);
int vmc_write_weights(const vmc_engine *e, const char *path, int digits);
/* FromFile::setupInitialWeights at any time: vmc_set_parameters from the file. */
int vmc_read_weights(vmc_engine *e, const char *path);
/* Walker state for an exact restart (no counterpart in the reference): the walkers'
 * records, running sums, Pade masks, Philox counters and status words, the
 * parameters, optimiser moments and step, and the refresh cadence, in a binary file.
 * Loading needs an engine created from the same input.in (same particles, walkers,
 * precision, elements); an engine resumed from a file continues exactly as the
 * saving engine would have. */
int vmc_save_state(const vmc_engine *e, const char *path);
int vmc_load_state(vmc_engine *e, const char *path);

/* ---- Multi-system batch (no counterpart in the reference) ----
 *
 * Many systems (quantum dots and atoms of different N, omega, Z), each with its
 * own input.in text, walker pool, parameters and optimiser, iterated together:
 * one persistent sweep kernel per round takes work items (a system's run of
 * walkers) from a queue ordered by cost, so large and small systems share the
 * GPU; every iteration is a captured CUDA graph (parameter upload, sweeps, FP64
 * refreshes, reductions, result download) replayed with the current parameters.
 * The CTA width (walkers per block) and work-item size are chosen by an
 * autotuner that times one iteration per candidate (the first iterations run
 * eagerly while it tunes).  Each system computes exactly what vmc_run_iteration
 * computes for it alone (the same walker streams, reductions and optimiser step).
 *
 * Systems: 2D closed-shell quantum dots with Slater(Hermite) x Gaussian x Pade,
 * Coulomb, importance sampling (all in the batch's precision and compat mode), and
 * general-path systems: hydrogen-orbital atoms with SimpleJastrow in the batch's
 * precision (mixed: the FP32 atom sweep with an FP64 Slater inverse, re-inverted in
 * FP64 after each round), other general-path systems (RBM, SimpleJastrow on other
 * bases) in FP64; not the MLP Jastrow.  Up to VMC_BATCH_MAX_SYSTEMS systems, at most
 * 16 of them on the general path; one batch per device at a time (its system table
 * is a device constant).  opt (may be NULL): device, compat and refresh_interval
 * apply to every system, precision to the dots and those atoms (NULL or -1: each
 * text's own); walker counts come from each text. */
#define VMC_BATCH_MAX_SYSTEMS 64
typedef struct vmc_batch vmc_batch;

typedef struct {
    int n_systems, n_general;
    long long n_walkers;        /* over all systems                                   */
    int precision;              /* of the dots                                        */
    int walkers_per_block;      /* chosen CTA width (warps), 0 while tuning            */
    int walkers_per_item;       /* chosen work-item size                              */
    int grid;                   /* persistent CTAs of the sweep                       */
    int tuned;                  /* 1 once the autotuner (or vmc_batch_set_tile) chose   */
    int graph_captures;         /* CUDA graphs captured so far                        */
    int graph_replay;           /* 1 if the last iteration replayed a captured graph   */
    int rounds;                 /* sweep launches of the last iteration               */
    double seconds;             /* device time of the last iteration                  */
    double sweep_seconds;       /* of its sweep launches                              */
    double walker_moves;        /* walker-moves of the last iteration                 */
} vmc_batch_info;

typedef struct {
    int walkers_per_block, walkers_per_item, grid;
    double ns_per_walker_move;  /* sweep time per walker-move of its trial iteration, or < 0 */
} vmc_batch_candidate;

int vmc_batch_create(const char *const *input_texts, int n_systems, const vmc_options *opt, vmc_batch **out);
void vmc_batch_destroy(vmc_batch *b);
int vmc_batch_get_info(const vmc_batch *b, vmc_batch_info *out);
/* The engine of system s (parameters, walkers, evaluation); owned by the batch. */
int vmc_batch_system(vmc_batch *b, int s, vmc_engine **engine);
/* vmc_init_walkers for every system; seeds: n_systems seeds, or NULL for each
 * system's configured seed. */
int vmc_batch_init_walkers(vmc_batch *b, const uint64_t *seeds);
/* Fix the tile instead of tuning (walkers_per_block 1..8, walkers_per_item >= 1). */
int vmc_batch_set_tile(vmc_batch *b, int walkers_per_block, int walkers_per_item);
/* One optimisation iteration of every system; out: n_systems averages (may be
 * NULL).  Each system's totals of the iteration: vmc_batch_last_sums. */
int vmc_batch_run_iteration(vmc_batch *b, int iteration, vmc_averages *out);
int vmc_batch_last_sums(const vmc_batch *b, vmc_sums *out /* n_systems */);
/* The autotuner's candidates and their timings; returns how many (<= n written). */
int vmc_batch_tuning(const vmc_batch *b, vmc_batch_candidate *out, int n);

/* ---- Allocation-free evaluation (no counterpart in the reference) ----
 *
 * Kinetic, external and interaction energy ({T, V_ext, V_int}, as vmc_eval's
 * `energies`) of n_walkers walkers at caller-given positions, in FP64, without
 * creating an engine and without allocating device memory.  For callers that
 * cannot allocate at that moment: a process whose device memory is held by
 * another framework's pool, a loop that must not stall other streams (freeing
 * device memory synchronises the device), code running while a stream is being
 * captured into a graph.
 *
 * input_in_text: the system as for vmc_create (numWalkers and precision are
 *   ignored); theta: host, n_elements x p_max row-major, the shape
 *   vmc_get_info reports; positions: device memory of the current device,
 *   n_walkers x (numParticles x numDimensions) doubles; energies: device memory
 *   of the current device, n_walkers x 3 doubles; stream: cudaStream_t (NULL =
 *   the default stream).  The work is enqueued on `stream` and the call returns
 *   without waiting: energies are valid once that work completes.  A walker
 *   whose Slater block is singular at its positions gets NaN energies.
 *
 * Every intermediate lives in one fixed device array of
 * VMC_NOALLOC_SCRATCH_BYTES per device (reserved when the library's module
 * loads); a walker count whose intermediates do not fit is rejected with
 * VMC_E_ARG and a message giving the largest count that fits (1,584 walkers
 * at 56 particles in 2D, 27,503 at 6).  All
 * calls share that array: calls whose GPU work overlaps (different streams or
 * host threads without ordering) race and corrupt each other's results, so
 * serialise them, e.g. on one stream.  The first call on each device looks up
 * the array's address and uploads the kernels' coefficient table with
 * synchronous copies: make it before any stream capture. */
#define VMC_NOALLOC_SCRATCH_BYTES (32u << 20)
int vmc_local_energies_noalloc(const char *input_in_text, const double *theta, int n_elements,
                               int p_max, const double *positions, int n_walkers,
                               double *energies, void *stream);

#ifdef __cplusplus
}
#endif
#endif

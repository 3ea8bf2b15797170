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

#define VMC_ABI_VERSION 2

enum {
    VMC_OK = 0,
    VMC_E_CONFIG = -1,      /* input.in error: unknown key, bad value (parser.cpp:314-320 aborts) */
    VMC_E_UNSUPPORTED = -2, /* a configuration the engine does not implement                   */
    VMC_E_CUDA = -3,        /* CUDA runtime error                                              */
    VMC_E_ARG = -4,         /* bad argument (size, NULL)                                       */
    VMC_E_NAN = -5,         /* NaN kinetic energy (sampler.cpp:219-225 aborts with 143)        */
    VMC_E_SINGULAR = -6,    /* singular Slater block at (re)initialisation                     */
    VMC_E_STATE = -7,       /* call out of order (e.g. sampling before walkers exist)          */
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
} vmc_info;

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

/* Version of this ABI, for a binding to check. */
int vmc_abi_version(void);

/* Parse input.in text and build an engine on a device.  Replaces
 * System::parser + System::initializeSystem (parser.cpp:25-333, system.cpp:50-73).
 * `opt` may be NULL.  Walkers are created by vmc_init_walkers. */
int vmc_create(const char *input_in_text, const vmc_options *opt, vmc_engine **out);
void vmc_destroy(vmc_engine *e);
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

/* Per-walker sampled-energy means of the last vmc_sample (W values). */
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

/* Per-walker status words (OR of VMC status bits) since creation. */
int vmc_get_status(const vmc_engine *e, uint32_t *status /* W */);

/* Full run as System::runSimulation (system.cpp:81-139) without terminal output:
 * numIterations iterations; per-iteration averages to `history` (may be NULL,
 * n_iterations entries). */
int vmc_run_simulation(vmc_engine *e, vmc_averages *history, int n_history);

/* Device-side stopwatch on the engine's stream: mode 0 records the start; mode 1
 * records the stop, waits for it and writes the elapsed milliseconds. */
int vmc_stopwatch(vmc_engine *e, int mode, double *ms);

/* FMA throughput of a device, FP32 (VMC_PRECISION_MIXED) or FP64, measured with a
 * register-resident loop over all SMs; TFLOP/s counting an FMA as 2 flops.  The
 * roofline denominator of the CUDA-core-bound sweep kernel. */
int vmc_measure_fma_peak(int device, int precision, double *tflops);

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

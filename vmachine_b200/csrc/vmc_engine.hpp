// Engine state shared by the host files of the library (vmc_engine.cu, vmc_batch.cu).
// Not part of the C ABI: callers see vmc_engine as an opaque handle.
#pragma once
#include <string>
#include <vector>

#include "vmc_b200.h"
#include "vmc_config.hpp"
#include "vmc_general.hpp"
#include "vmc_kernels.cuh"

namespace vmc {
int set_last_error(int code, const char *msg);
// identifier of the current CUDA context (0: unknown), for per-context set-up
unsigned long long current_context_id();
}  // namespace vmc

struct vmc_engine {
    using Config = vmc::Config;
    using Layout = vmc::Layout;
    using KernelSet = vmc::KernelSet;
    using GenParams = vmc::GenParams;
    Config cfg;
    int device = 0, num_sms = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    int W = 0, N = 0, dim = 0, D = 0, n_orb = 0, K = 0, E = 0, Pmax = 0, EP = 0, nacc = 0;
    // accumulators per walker on the device: nacc on the quantum-dot path; on the
    // general path 9 + 2 x the active parameters (act, no padding, no MLP row)
    int nacc_dev = 0;
    std::vector<int> act;
    int *d_act = nullptr;
    int precision = 0, compat = 1, flags = 0, sampling = 0;
    int steps_per_walker = 0, burn_in = 0, batches = 1;
    int wpb = 0, refresh_interval = 0, sweep_chunk = 2048;
    bool owner = false;  // production dot sweep in the owner form (vmc_owner_sweep.cuh)
    bool refresh_auto = false;          // refreshInterval: auto (mixed precision)
    double drift_tol = 1e-4;            // inverse drift that halves the interval
    size_t elem_bytes = 8;
    Layout L{};
    KernelSet ks;
    // general path (SimpleJastrow, RBM, hydrogen orbitals): FP64 kernels of vmc_general.cu
    bool general = false;
    GenParams gen{};
    double *d_theta = nullptr;  // E x p_max on the device (general path)
    // MLP Jastrow: bf16-rounded weights, parameter-gradient snapshots and sums
    int mlp_e = -1;                // element index, or -1
    float *d_mlpw = nullptr;
    float *d_mlp_cache = nullptr;  // MLP Jastrow dot: per-walker pair and one-body caches
    float *d_snap_x = nullptr;
    double *d_snap_e = nullptr, *d_mlp_out = nullptr;
    size_t snap_cap = 0;           // snapshots the buffers hold
    std::vector<double> theta;
    double gamma_prev = 0.0;
    bool have_walkers = false;
    unsigned long long seed = 0;
    // optimiser state (adam.cpp:12-37, gradientdescent.cpp/sgd.cpp)
    std::vector<double> opt_m, opt_v;
    int opt_step = 0;
    // device buffers
    void *d_state = nullptr;
    double *d_scal = nullptr, *d_acc = nullptr, *d_out = nullptr, *d_drift = nullptr, *d_wmean = nullptr;
    unsigned long long *d_mask = nullptr, *d_counter = nullptr;
    unsigned *d_status = nullptr;
    double *d_pos = nullptr;  // W x D positions staged for the host link
    std::vector<cudaEvent_t> sweep_events;  // per-launch timing of the sweep kernel
    cudaEvent_t sw0 = nullptr, sw1 = nullptr;  // vmc_stopwatch
    // optional per-step energy record of vmc_sample: (T, V_ext, V_int) of every walker
    // and step, W x rec_stride x 3 (the blocking analysis)
    double *d_rec = nullptr;
    int rec_stride = 0;
    // optional electron-density histograms filled by vmc_sample (dens_bins > 0)
    unsigned long long *d_dens_radial = nullptr, *d_dens_grid = nullptr, *d_dens_pair = nullptr;
    int dens_bins = 0;
    double dens_step = 0.0, dens_max = 0.0;
    // blocking of the last vmc_run_simulation's final iteration (doResampling)
    vmc_blocking_result final_blocking{};
    bool have_final = false;
    // optional replayed random stream consumed by vmc_sample (W x replay_len x 3)
    double *d_replay = nullptr;
    int replay_len = 0, replay_pos = 0;
    // last sampling pass
    vmc_sums last{};
    double last_samples_per_walker = 0.0;
    double last_walker_std_error = 0.0;
};

namespace vmc {

// Longest FP64 refresh interval the drift autotuner may choose for any system.
constexpr int REFRESH_CAP_MIN = 8192;
// Device memory vmc_run_simulation may spend on the last iteration's energy record,
// and the most lines it writes to the instant-energy file.
constexpr double FINAL_RECORD_BYTES = 16.0e9;
constexpr double INSTANT_FILE_LINES = 1.0e8;

// Coefficients of the normalised Hermite recurrence (each kernel unit holds a copy
// in constant memory).
HermiteCoef hermite_coefficients();
// Kernel parameters of the engine's current state (parameters, gamma history,
// device buffers).
// the owner-form sweep's per-launch constants (SweepArgs::oc, ocf) from a.P
void owner_constants(const vmc_engine *e, SweepArgs &a);
Params engine_params(const vmc_engine *e);
// Shared bytes per warp of the sweep (the staged record, Pade mask and scalars) and
// of the FP64 rebuild.
int engine_sweep_smem_per_warp(const vmc_engine *e);
int engine_rebuild_smem_per_warp(const vmc_engine *e);
// FP64 re-derivation of every walker's state from its positions (the periodic
// refresh, drift into drift[w] when non-null), on the engine's stream.
int engine_refresh(vmc_engine *e, double *drift);

// One sampling pass as reduced on the device, turned into the engine's results by
// finish_sample (the tail of vmc_sample): totals, the refresh cadence, the
// last-pass record, and `sums` = the nacc accumulators in (element, parameter) order.
struct SamplePass {
    int steps, burn_in, bs, n_launch, n_refresh;
    const double *dev_sums;        // nacc_dev reduced accumulators
    unsigned status;               // OR of the walkers' status words
    std::vector<double> *drift;    // per-walker inverse drift of the refreshes, or null
    double ms, sweep_ms;           // device time of the pass and of its sweep launches
    double walker_std_error;       // < 0: computed from the accumulators here
};
int finish_sample(vmc_engine *e, const SamplePass &p, vmc_sums *out, std::vector<double> &sums);
// vmc_apply_sums; with refresh = false the walkers are not re-derived for the new
// parameters (the caller does it, e.g. inside a captured multi-system iteration).
int apply_sums(vmc_engine *e, const vmc_sums *total, const double *grad_sum, const double *egrad_sum,
               vmc_averages *out, bool refresh);
// vmc_set_parameters with the same refresh switch.
int set_parameters(vmc_engine *e, const double *theta, bool refresh);
// The host parameters to the device copies the kernels read (general path, MLP
// weights); the walkers are not re-derived.
int upload_parameters(vmc_engine *e);
// Parameter files in the reference's text format (vmc_checkpoint.cu): read E x P
// values ("" or why not); write with `digits` significant digits.
std::string read_weights_file(const std::string &path, int E, int P, std::vector<double> &theta);
int write_weights_file(const vmc_engine *e, const std::string &path, int digits);
// Electron-density histograms of the following vmc_sample calls (vmc_density.cu):
// begin allocates and zeroes them, end copies them out (null: skip) and frees them.
int density_begin(vmc_engine *e, int bins, double max_radius, bool radial, bool spatial, bool pair);
int density_end(vmc_engine *e, uint64_t *radial, uint64_t *spatial, uint64_t *pair);
// Integer counts as the reference prints Eigen integer vectors and matrices.
int write_counts(const std::string &path, const uint64_t *v, int rows, int cols);
// Blocking of an energy record of `steps` steps per walker (vmc_blocking.cu).
int block_record(vmc_engine *e, const double *rec, int steps, int burn_in, vmc_blocking_result *out);

}  // namespace vmc

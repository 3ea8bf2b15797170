// Host side of the multi-system batch (vmc_batch_* in include/vmc_b200.h).
//
// Every system is an ordinary engine (vmc_create from its own input.in text) whose
// stream is the batch's; the batch owns the iteration: it writes the systems'
// kernel arguments to pinned memory, replays one captured CUDA graph per schedule
// (argument upload into the constant-memory system table, accumulator clear,
// parameter refresh, the persistent sweep of each round with the FP64 refresh after
// it, the per-system reductions and the download of the totals), then finishes each
// system's sampling pass and optimiser step on the host exactly as vmc_sample and
// vmc_apply_sums do for one engine.
//
// Work items and the tile.  Items are runs of `per_item` walkers of one system
// (`per_item` pairs for the dots of at most three shells, whose warps carry two
// walkers), ordered by decreasing walker-steps x cost per step; the autotuner times one
// iteration per (walkers per block, walkers per item) candidate and keeps the
// fastest; the graph is re-captured when the schedule (rounds, refresh rounds,
// tile) changes, e.g. while the refresh intervals settle.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <string>
#include <vector>

#include "vmc_batch_kernels.cuh"
#include "vmc_engine.hpp"

namespace vmc {
BatchOps batch_ops_f32();
BatchOps batch_ops_f64();
}  // namespace vmc

using namespace vmc;

struct vmc_batch {
    int device = 0, num_sms = 0, precision = VMC_PRECISION_FP64, compat = -1;
    cudaStream_t stream = nullptr;
    std::vector<vmc_engine *> sys;
    std::vector<int> kind, gen_of;  // per system: Hermite shells or BATCH_GENERAL; index into gen
    std::vector<double> cost;       // work per walker-step (ordering only)
    std::vector<char> theta_dirty;  // parameters changed since the last sweep
    // per system: the rounds after which an FP32 general-path system (the atoms in mixed
    // precision) takes its FP64 re-inversion, this iteration
    std::vector<int> gen_rounds;
    int n_gen = 0;
    BatchOps ops{};
    const void *sweep_fn = nullptr;
    int sweep_smem = 0, rebuild_smem = 0;  // shared bytes per warp
    int max_nacc = 0, stride = 0, queue_cap = 0;
    long long total_walkers = 0;
    bool any_refresh = false;
    // work items of the current per_item
    int2 *d_items = nullptr;
    int n_items = 0, items_per = 0, items_cap = 0;
    int *d_queue = nullptr;
    double *d_out = nullptr, *d_drift_all = nullptr;
    long long *d_drift_off = nullptr;
    std::vector<long long> drift_off;
    // pinned host mirrors
    BatchSys *h_sys = nullptr;
    GenParams *h_gen = nullptr;
    double *h_out = nullptr, *h_drift = nullptr;
    // tile candidates
    struct Cand {
        int wpb, per_item, grid;
        double ns = -1.0;
    };
    std::vector<Cand> cands;
    int next_cand = 0, chosen = -1, rebuild_grid = 0;
    // captured iteration
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    std::vector<long long> key;
    int captures = 0;
    bool last_replay = false;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<cudaEvent_t> sev;  // start / end of each round's sweep
    // last iteration
    int last_rounds = 0;
    double last_ms = 0.0, last_sweep_ms = 0.0, last_moves = 0.0;
    std::vector<vmc_sums> last;
};

namespace {

std::mutex g_batch_mu;
bool g_batch_on_device[64] = {false};  // one batch per device: the system table is a device constant

int bfail(int code, const std::string &m) { return set_last_error(code, m.c_str()); }

#define BCUDA(expr)                                                                          \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess) return bfail(VMC_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    } while (0)

// Work per walker-step, for ordering the items: the dot sweep's algorithmic flops
// (Hermite tables, Slater ratio row, Sherman-Morrison, derivative refresh, pair and
// kinetic terms); a general-path step (FP64, record in HBM) weighted 8x its pair,
// orbital and coordinate work.
double step_cost(const vmc_engine *e, int kind)
{
    const double N = e->N, n = e->n_orb, d = e->dim, K = std::max(kind, 1);
    if (kind == BATCH_GENERAL) return 8.0 * (N * N * 16 + n * n * 8 + N * d * 32 + e->EP * 4);
    const double tables = d * 4 * (K - 1);
    return tables + n * (2 * n + 2 * K) + 2 * n * n + n * (tables + 4 * n + 3 * d * (2 * K - 3)) +
           (N - 1) * (10 * d + 38) + 7 * N * d + 40;
}

void free_batch(vmc_batch *b)
{
    if (!b) return;
    cudaSetDevice(b->device);
    if (b->stream) cudaStreamSynchronize(b->stream);
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->graph) cudaGraphDestroy(b->graph);
    for (vmc_engine *e : b->sys) {
        if (e->stream == b->stream) e->stream = nullptr;  // the batch's stream, destroyed below
        vmc_destroy(e);
    }
    cudaFree(b->d_items);
    cudaFree(b->d_queue);
    cudaFree(b->d_out);
    cudaFree(b->d_drift_all);
    cudaFree(b->d_drift_off);
    cudaFreeHost(b->h_sys);
    cudaFreeHost(b->h_gen);
    cudaFreeHost(b->h_out);
    cudaFreeHost(b->h_drift);
    for (cudaEvent_t ev : b->sev) cudaEventDestroy(ev);
    if (b->ev0) cudaEventDestroy(b->ev0);
    if (b->ev1) cudaEventDestroy(b->ev1);
    if (b->stream) cudaStreamDestroy(b->stream);
    {
        std::lock_guard<std::mutex> lk(g_batch_mu);
        if (b->device >= 0 && b->device < 64) g_batch_on_device[b->device] = false;
    }
    delete b;
}

// Walkers per warp of a system in the batch sweep: the engine's choice for the dots
// up to N = 30 (Hermite shells K <= 5) and for the general path's small atoms, one
// otherwise (the batch kernel carries the several-walker forms only for those).
static int batch_walkers_per_warp(const vmc_engine *e, int kind)
{
    if (e->general) return e->gen.variant == GV_ATOM ? e->gen.seg : 1;
    return (kind >= 1 && kind <= 5) ? e->ks.seg : 1;
}

// Items of per_item walkers, longest work first (ties: system order, then walker).
int build_items(vmc_batch *b, int per_item)
{
    if (b->items_per == per_item && b->d_items) return VMC_OK;
    struct It {
        double c;
        int s, w0;
    };
    std::vector<It> v;
    for (size_t s = 0; s < b->sys.size(); ++s) {
        const vmc_engine *e = b->sys[s];
        // an item is per_item warps' worth: per_item walkers, or pairs for two-walker warps
        const double c = b->cost[s] * (double)(e->steps_per_walker + e->burn_in) * per_item;
        const int width = per_item * batch_walkers_per_warp(e, b->kind[s]);
        for (int w0 = 0; w0 < e->W; w0 += width) v.push_back({c, (int)s, w0});
    }
    std::stable_sort(v.begin(), v.end(), [](const It &x, const It &y) { return x.c > y.c; });
    std::vector<int2> items(v.size());
    for (size_t i = 0; i < v.size(); ++i) items[i] = make_int2(v[i].s, v[i].w0);
    if ((int)items.size() > b->items_cap) {
        cudaFree(b->d_items);
        b->d_items = nullptr;
        BCUDA(cudaMalloc(&b->d_items, items.size() * sizeof(int2)));
        b->items_cap = (int)items.size();
    }
    BCUDA(cudaMemcpyAsync(b->d_items, items.data(), items.size() * sizeof(int2), cudaMemcpyHostToDevice, b->stream));
    BCUDA(cudaStreamSynchronize(b->stream));
    b->n_items = (int)items.size();
    b->items_per = per_item;
    return VMC_OK;
}

int launch(const void *fn, dim3 grid, dim3 block, size_t smem, cudaStream_t st, void **args)
{
    BCUDA(cudaLaunchKernel(fn, grid, block, args, smem, st));
    return VMC_OK;
}

int record(cudaEvent_t ev, cudaStream_t st, bool capturing)
{
    if (capturing) BCUDA(cudaEventRecordWithFlags(ev, st, cudaEventRecordExternal));
    else BCUDA(cudaEventRecord(ev, st));
    return VMC_OK;
}

// The iteration's device work on the batch stream (captured or eager).
int enqueue(vmc_batch *b, const vmc_batch::Cand &c, int rounds, const std::vector<char> &rebuild_round,
            bool theta_refresh, bool capturing)
{
    const int n = (int)b->sys.size();
    cudaStream_t st = b->stream;
    BCUDA(b->ops.upload(b->h_sys, n, b->h_gen, b->n_gen, st));
    BCUDA(cudaMemsetAsync(b->d_queue, 0, (size_t)(2 * rounds + 1) * sizeof(int), st));
    int rc = launch(b->ops.clear, dim3(32, n), dim3(256), 0, st, nullptr);
    if (rc) return rc;
    const int rb_smem = 4 * b->rebuild_smem;
    if (theta_refresh) {
        BatchLaunch L{b->d_items, b->n_items, b->items_per, b->d_queue + 2 * rounds, -1, b->rebuild_smem};
        void *args[] = {&L};
        if ((rc = launch(b->ops.rebuild, dim3(b->rebuild_grid), dim3(128), rb_smem, st, args))) return rc;
    }
    for (int r = 0; r < rounds; ++r) {
        if ((rc = record(b->sev[2 * r], st, capturing))) return rc;
        BatchLaunch L{b->d_items, b->n_items, b->items_per, b->d_queue + 2 * r, r, b->sweep_smem};
        void *args[] = {&L};
        if ((rc = launch(b->sweep_fn, dim3(c.grid), dim3(32 * c.wpb), (size_t)c.wpb * b->sweep_smem, st, args)))
            return rc;
        if ((rc = record(b->sev[2 * r + 1], st, capturing))) return rc;
        if (rebuild_round[r]) {
            BatchLaunch R{b->d_items, b->n_items, b->items_per, b->d_queue + 2 * r + 1, r, b->rebuild_smem};
            void *rargs[] = {&R};
            if ((rc = launch(b->ops.rebuild, dim3(b->rebuild_grid), dim3(128), rb_smem, st, rargs))) return rc;
        }
        // the FP32 atoms: FP64 re-inversion and evaluation after each of their launches
        for (int s = 0; s < n; ++s)
            if (b->gen_rounds[s] > r) {
                vmc_engine *e = b->sys[s];
                BCUDA(gen_launch_state(engine_params(e), e->gen, GEN_REFRESH, nullptr, nullptr, nullptr, nullptr, st));
            }
    }
    double *out = b->d_out, *drift = b->d_drift_all;
    long long *doff = b->d_drift_off;
    int stride = b->stride;
    void *rargs[] = {&out, &stride, &drift, &doff};
    if ((rc = launch(b->ops.reduce, dim3(b->max_nacc + 1, n), dim3(256), 0, st, rargs))) return rc;
    BCUDA(cudaMemcpyAsync(b->h_out, b->d_out, (size_t)n * b->stride * sizeof(double), cudaMemcpyDeviceToHost, st));
    if (b->any_refresh)
        BCUDA(cudaMemcpyAsync(b->h_drift, b->d_drift_all, (size_t)b->total_walkers * sizeof(double),
                              cudaMemcpyDeviceToHost, st));
    return VMC_OK;
}

int tile_candidates(vmc_batch *b)
{
    const int max_wpb = b->precision == VMC_PRECISION_MIXED ? 8 : 4;  // the sweep's launch bounds
    for (int wpb : {8, 4, 2}) {
        if (wpb > max_wpb) continue;
        const size_t smem = (size_t)wpb * b->sweep_smem;
        if (smem > 227 * 1024) continue;
        BCUDA(cudaFuncSetAttribute(b->sweep_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        int blocks = 0;
        BCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&blocks, b->sweep_fn, 32 * wpb, smem));
        if (blocks < 1) continue;
        for (int per_item : {1, 4}) b->cands.push_back({wpb, per_item, blocks * b->num_sms});
    }
    if (b->cands.empty()) return bfail(VMC_E_UNSUPPORTED, "no tile fits the batch's largest walker record");
    // launches take up to the widest candidate's shared memory
    int widest = 0;
    for (const vmc_batch::Cand &c : b->cands) widest = std::max(widest, c.wpb);
    BCUDA(cudaFuncSetAttribute(b->sweep_fn, cudaFuncAttributeMaxDynamicSharedMemorySize, widest * b->sweep_smem));
    const size_t rsmem = (size_t)4 * b->rebuild_smem;
    BCUDA(cudaFuncSetAttribute(b->ops.rebuild, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)std::max<size_t>(rsmem, 1)));
    int rblocks = 0;
    BCUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&rblocks, b->ops.rebuild, 128, rsmem));
    b->rebuild_grid = std::max(1, rblocks) * b->num_sms;
    return VMC_OK;
}

}  // namespace

extern "C" {

int vmc_batch_create(const char *const *texts, int n_systems, const vmc_options *opt, vmc_batch **out)
{
    if (!texts || !out) return bfail(VMC_E_ARG, "null argument");
    *out = nullptr;
    if (n_systems < 1 || n_systems > BATCH_MAX_SYS)
        return bfail(VMC_E_ARG, "a batch holds 1 to " + std::to_string(BATCH_MAX_SYS) + " systems");
    vmc_options o{};
    o.device = 0;
    o.precision = -1;
    o.num_walkers = -1;
    o.walkers_per_block = -1;
    o.refresh_interval = -1;
    o.compat = -1;
    if (opt) {
        o.device = opt->device;
        o.precision = opt->precision;
        o.refresh_interval = opt->refresh_interval;
        o.compat = opt->compat;
    }
    if (o.device < 0 || o.device >= 64) return bfail(VMC_E_ARG, "bad device");
    {
        std::lock_guard<std::mutex> lk(g_batch_mu);
        if (g_batch_on_device[o.device]) return bfail(VMC_E_STATE, "a batch already exists on this device");
        g_batch_on_device[o.device] = true;
    }
    vmc_batch *b = new vmc_batch();
    b->device = o.device;
    auto reject = [&](int code, const std::string &m) {
        free_batch(b);
        return bfail(code, m);
    };
    int dot_precision = -1;
    for (int s = 0; s < n_systems; ++s) {
        if (!texts[s]) return reject(VMC_E_ARG, "null input text");
        vmc_engine *e = nullptr;
        int rc = vmc_create(texts[s], &o, &e);
        if (rc == VMC_E_UNSUPPORTED && o.precision == VMC_PRECISION_MIXED) {
            // a general-path system runs in FP64 whatever the dots' precision
            vmc_options o64 = o;
            o64.precision = VMC_PRECISION_FP64;
            vmc_engine *e64 = nullptr;
            if (vmc_create(texts[s], &o64, &e64) == VMC_OK) {
                if (e64->general) {
                    e = e64;
                    rc = VMC_OK;
                } else {
                    vmc_destroy(e64);
                }
            }
        }
        if (rc) {
            const std::string why = vmc_last_error();
            return reject(rc, "system " + std::to_string(s) + ": " + why);
        }
        b->sys.push_back(e);
        int kind;
        if (e->general) {
            if (e->mlp_e >= 0) return reject(VMC_E_UNSUPPORTED, "system " + std::to_string(s) + ": the MLP Jastrow runs alone");
            if (b->n_gen >= BATCH_MAX_GEN)
                return reject(VMC_E_UNSUPPORTED, "more than " + std::to_string(BATCH_MAX_GEN) + " general-path systems");
            kind = BATCH_GENERAL;
            b->gen_of.push_back(b->n_gen++);
        } else {
            const bool dot = e->dim == 2 && e->K >= 1 && e->K <= 7 &&
                             (e->flags == FX_DOT_COMPAT || e->flags == FX_DOT_CORRECTED);
            if (!dot)
                return reject(VMC_E_UNSUPPORTED, "system " + std::to_string(s) +
                                                     ": the batch takes 2D closed-shell dots (Slater x Gaussian x "
                                                     "Pade, Coulomb, importance sampling) and general-path systems");
            if (dot_precision >= 0 && e->precision != dot_precision)
                return reject(VMC_E_UNSUPPORTED, "the batch's dots must share one precision");
            if (b->compat >= 0 && e->compat != b->compat)
                return reject(VMC_E_UNSUPPORTED, "the batch's dots must share one compat mode");
            dot_precision = e->precision;
            b->compat = e->compat;
            kind = e->K;
            b->gen_of.push_back(-1);
        }
        b->kind.push_back(kind);
        b->cost.push_back(step_cost(e, kind));
        b->theta_dirty.push_back(0);
        b->max_nacc = std::max(b->max_nacc, e->nacc_dev);
        b->drift_off.push_back(b->total_walkers);
        b->total_walkers += e->W;
        if (!e->general && e->refresh_interval > 0) b->any_refresh = true;
        if (!e->general)
            b->rebuild_smem = std::max(b->rebuild_smem, engine_rebuild_smem_per_warp(e));
        b->sweep_smem = std::max(b->sweep_smem, e->general ? (int)(GEN_SCR * sizeof(double))
                                                           : batch_walkers_per_warp(e, kind) * engine_sweep_smem_per_warp(e));
        // N = 42 and 56 run the owner-form sweep in the batch too (as they do alone)
        if (!e->general && e->owner) b->sweep_smem = std::max(b->sweep_smem, e->ks.owner_smem);
    }
    if (dot_precision < 0)  // general-path systems only: slices as large as their staging
        for (vmc_engine *e : b->sys)
            b->sweep_smem = std::max(b->sweep_smem,
                                     (int)((GEN_SCR + gen_stage_doubles(e->gen, e->nacc_dev)) * sizeof(double)));
    b->precision = dot_precision >= 0 ? dot_precision : VMC_PRECISION_FP64;
    if (b->compat < 0) b->compat = b->sys[0]->compat;
    b->stride = b->max_nacc + BATCH_EXTRA;
    b->ops = b->precision == VMC_PRECISION_MIXED ? batch_ops_f32() : batch_ops_f64();
    b->sweep_fn = b->compat ? b->ops.sweep_compat : b->ops.sweep_corrected;
    b->last.resize(n_systems);
    int rc = [&]() -> int {
        BCUDA(cudaSetDevice(b->device));
        BCUDA(cudaDeviceSynchronize());  // the engines' own streams are done with their set-up
        BCUDA(cudaDeviceGetAttribute(&b->num_sms, cudaDevAttrMultiProcessorCount, b->device));
        BCUDA(cudaStreamCreateWithFlags(&b->stream, cudaStreamNonBlocking));
        for (vmc_engine *e : b->sys) {
            cudaStreamDestroy(e->stream);
            e->stream = b->stream;
        }
        BCUDA(b->ops.upload_hermite(hermite_coefficients()));
        BCUDA(cudaEventCreate(&b->ev0));
        BCUDA(cudaEventCreate(&b->ev1));
        // rounds: at most steps / (smallest refresh interval) per system
        int cap = 1;
        for (vmc_engine *e : b->sys) {
            const int steps = e->steps_per_walker + e->burn_in;
            // general-path systems run in launches of sweep_chunk steps (the FP32 atoms
            // re-invert in FP64 after each)
            const int chunk_min = e->general ? e->sweep_chunk
                                  : e->refresh_auto ? e->D
                                  : e->refresh_interval > 0 ? e->refresh_interval : e->sweep_chunk;
            cap = std::max(cap, (steps + chunk_min - 1) / chunk_min);
        }
        b->queue_cap = cap;
        BCUDA(cudaMalloc(&b->d_queue, (size_t)(2 * cap + 1) * sizeof(int)));
        BCUDA(cudaMalloc(&b->d_out, (size_t)n_systems * b->stride * sizeof(double)));
        BCUDA(cudaMalloc(&b->d_drift_all, (size_t)b->total_walkers * sizeof(double)));
        BCUDA(cudaMalloc(&b->d_drift_off, (size_t)n_systems * sizeof(long long)));
        BCUDA(cudaMemcpy(b->d_drift_off, b->drift_off.data(), n_systems * sizeof(long long), cudaMemcpyHostToDevice));
        BCUDA(cudaHostAlloc(&b->h_sys, sizeof(BatchSys) * BATCH_MAX_SYS, cudaHostAllocDefault));
        BCUDA(cudaHostAlloc(&b->h_gen, sizeof(GenParams) * BATCH_MAX_GEN, cudaHostAllocDefault));
        BCUDA(cudaHostAlloc(&b->h_out, (size_t)n_systems * b->stride * sizeof(double), cudaHostAllocDefault));
        BCUDA(cudaHostAlloc(&b->h_drift, (size_t)b->total_walkers * sizeof(double), cudaHostAllocDefault));
        std::memset(b->h_sys, 0, sizeof(BatchSys) * BATCH_MAX_SYS);
        std::memset(b->h_gen, 0, sizeof(GenParams) * BATCH_MAX_GEN);
        b->sev.resize(2 * cap);
        for (cudaEvent_t &ev : b->sev) BCUDA(cudaEventCreate(&ev));
        return tile_candidates(b);
    }();
    if (rc) {
        const std::string why = vmc_last_error();
        free_batch(b);
        return bfail(rc, why);
    }
    *out = b;
    return VMC_OK;
}

void vmc_batch_destroy(vmc_batch *b) { free_batch(b); }

int vmc_batch_get_info(const vmc_batch *b, vmc_batch_info *o)
{
    if (!b || !o) return bfail(VMC_E_ARG, "null argument");
    std::memset(o, 0, sizeof(*o));
    o->n_systems = (int)b->sys.size();
    o->n_general = b->n_gen;
    o->n_walkers = b->total_walkers;
    o->precision = b->precision;
    if (b->chosen >= 0) {
        const vmc_batch::Cand &c = b->cands[b->chosen];
        o->walkers_per_block = c.wpb;
        o->walkers_per_item = c.per_item;
        o->grid = c.grid;
        o->tuned = 1;
    }
    o->graph_captures = b->captures;
    o->graph_replay = b->last_replay ? 1 : 0;
    o->rounds = b->last_rounds;
    o->seconds = b->last_ms * 1e-3;
    o->sweep_seconds = b->last_sweep_ms * 1e-3;
    o->walker_moves = b->last_moves;
    return VMC_OK;
}

int vmc_batch_system(vmc_batch *b, int s, vmc_engine **engine)
{
    if (!b || !engine) return bfail(VMC_E_ARG, "null argument");
    if (s < 0 || s >= (int)b->sys.size()) return bfail(VMC_E_ARG, "no such system");
    *engine = b->sys[s];
    return VMC_OK;
}

int vmc_batch_init_walkers(vmc_batch *b, const uint64_t *seeds)
{
    if (!b) return bfail(VMC_E_ARG, "null argument");
    for (size_t s = 0; s < b->sys.size(); ++s) {
        vmc_engine *e = b->sys[s];
        const int rc = vmc_init_walkers(e, nullptr, seeds ? seeds[s] : e->seed);
        if (rc) return rc;
        b->theta_dirty[s] = 0;
    }
    return VMC_OK;
}

int vmc_batch_set_tile(vmc_batch *b, int wpb, int per_item)
{
    if (!b) return bfail(VMC_E_ARG, "null argument");
    if (per_item < 1) return bfail(VMC_E_ARG, "walkers_per_item must be >= 1");
    for (size_t i = 0; i < b->cands.size(); ++i)
        if (b->cands[i].wpb == wpb) {
            vmc_batch::Cand c = b->cands[i];
            c.per_item = per_item;
            c.ns = -1.0;
            b->cands.push_back(c);
            b->chosen = (int)b->cands.size() - 1;
            return VMC_OK;
        }
    return bfail(VMC_E_ARG, "walkers_per_block not available for this batch (shared memory or precision)");
}

int vmc_batch_run_iteration(vmc_batch *b, int iteration, vmc_averages *avg)
{
    if (!b) return bfail(VMC_E_ARG, "null argument");
    BCUDA(cudaSetDevice(b->device));
    const int n = (int)b->sys.size();
    for (vmc_engine *e : b->sys)
        if (!e->have_walkers) return bfail(VMC_E_STATE, "vmc_batch_init_walkers first");
    // ---- schedule and arguments of every system
    int rounds = 0, rc = 0;
    bool theta_refresh = false;
    std::vector<int> n_launch(n);
    for (int s = 0; s < n; ++s) {
        vmc_engine *e = b->sys[s];
        const int steps = e->steps_per_walker + e->burn_in, burn = e->burn_in;
        const int chunk = e->general ? e->sweep_chunk : e->refresh_interval > 0 ? e->refresh_interval : e->sweep_chunk;
        n_launch[s] = (steps + chunk - 1) / chunk;
        rounds = std::max(rounds, n_launch[s]);
        const int bs = (steps - burn) / e->batches, m = iteration % e->batches;
        BatchSys &h = b->h_sys[s];
        h = BatchSys{};
        h.a.P = engine_params(e);
        h.a.steps = chunk;
        h.a.burn_in = burn;
        h.a.win_lo = bs * m;
        h.a.win_hi = bs * (m + 1);
        h.a.seed = e->seed;
        h.total_steps = steps;
        h.kind = b->kind[s];
        h.gen = std::max(0, b->gen_of[s]);
        h.refresh = (b->kind[s] != BATCH_GENERAL && e->refresh_interval > 0) ? 1 : 0;
        h.theta_refresh = (b->kind[s] != BATCH_GENERAL && b->theta_dirty[s]) ? 1 : 0;
        h.samples = steps - burn;
        h.seg = batch_walkers_per_warp(e, b->kind[s]);
        h.owner = (b->kind[s] == 6 || b->kind[s] == 7) && e->owner ? 1 : 0;
        if (h.owner) owner_constants(e, h.a);
        h.drift = e->d_drift;
        theta_refresh |= h.theta_refresh != 0;
        if (b->kind[s] == BATCH_GENERAL) {
            b->h_gen[b->gen_of[s]] = e->gen;
            if (b->theta_dirty[s] && (rc = engine_refresh(e, nullptr))) return rc;  // new parameters
        }
    }
    if (rounds > b->queue_cap) return bfail(VMC_E_STATE, "refresh schedule beyond the batch's queue");
    std::vector<char> rebuild_round(rounds, 0);
    for (int s = 0; s < n; ++s)
        if (b->h_sys[s].refresh)
            for (int r = 0; r < n_launch[s]; ++r) rebuild_round[r] = 1;
    b->gen_rounds.assign(n, 0);
    for (int s = 0; s < n; ++s)
        if (b->kind[s] == BATCH_GENERAL && b->sys[s]->gen.f32) b->gen_rounds[s] = n_launch[s];
    const bool tuning = b->chosen < 0;
    const vmc_batch::Cand c = tuning ? b->cands[b->next_cand % b->cands.size()] : b->cands[b->chosen];
    if ((rc = build_items(b, c.per_item))) return rc;
    // ---- replay the captured iteration (captured again when the schedule changed)
    if (!tuning) {
        std::vector<long long> key = {rounds, c.wpb, c.per_item, c.grid, b->n_items, theta_refresh ? 1 : 0,
                                      (long long)(size_t)b->d_items};
        for (char f : rebuild_round) key.push_back(f);
        for (int g : b->gen_rounds) key.push_back(g);
        if (key != b->key || !b->exec) {
            if (b->exec) cudaGraphExecDestroy(b->exec);
            if (b->graph) cudaGraphDestroy(b->graph);
            b->exec = nullptr;
            b->graph = nullptr;
            BCUDA(cudaStreamBeginCapture(b->stream, cudaStreamCaptureModeThreadLocal));
            rc = enqueue(b, c, rounds, rebuild_round, theta_refresh, true);
            cudaGraph_t g = nullptr;
            const cudaError_t ce = cudaStreamEndCapture(b->stream, &g);
            if (rc) {
                if (g) cudaGraphDestroy(g);
                return rc;
            }
            BCUDA(ce);
            b->graph = g;
            BCUDA(cudaGraphInstantiate(&b->exec, b->graph, 0));
            b->key = key;
            ++b->captures;
        }
        BCUDA(cudaEventRecord(b->ev0, b->stream));
        BCUDA(cudaGraphLaunch(b->exec, b->stream));
        BCUDA(cudaEventRecord(b->ev1, b->stream));
    } else {
        BCUDA(cudaEventRecord(b->ev0, b->stream));
        if ((rc = enqueue(b, c, rounds, rebuild_round, theta_refresh, false))) return rc;
        BCUDA(cudaEventRecord(b->ev1, b->stream));
    }
    b->last_replay = !tuning;
    BCUDA(cudaStreamSynchronize(b->stream));
    float ms = 0.f;
    BCUDA(cudaEventElapsedTime(&ms, b->ev0, b->ev1));
    double sweep_ms = 0.0, moves = 0.0;
    for (int r = 0; r < rounds; ++r) {
        float t = 0.f;
        BCUDA(cudaEventElapsedTime(&t, b->sev[2 * r], b->sev[2 * r + 1]));
        sweep_ms += t;
    }
    for (vmc_engine *e : b->sys) moves += (double)e->W * (e->steps_per_walker + e->burn_in);
    b->last_rounds = rounds;
    b->last_ms = ms;
    b->last_sweep_ms = sweep_ms;
    b->last_moves = moves;
    if (tuning) {
        // two passes over the candidates (the refresh intervals still settle in the
        // first iterations, changing the rounds); each keeps its better time
        vmc_batch::Cand &t = b->cands[b->next_cand % b->cands.size()];
        const double ns = sweep_ms * 1e6 / moves;
        t.ns = t.ns < 0 ? ns : std::min(t.ns, ns);
        if (++b->next_cand == 2 * (int)b->cands.size()) {
            int best = 0;
            for (int i = 1; i < (int)b->cands.size(); ++i)
                if (b->cands[i].ns < b->cands[best].ns) best = i;
            b->chosen = best;
        }
    }
    // ---- finish every system as vmc_sample + vmc_apply_sums would
    int first_err = 0;
    std::string first_msg;
    for (int s = 0; s < n; ++s) {
        vmc_engine *e = b->sys[s];
        const double *o = b->h_out + (size_t)s * b->stride;
        const double *x = o + b->stride - BATCH_EXTRA;
        const int steps = e->steps_per_walker + e->burn_in;
        std::vector<double> drift;
        if (b->h_sys[s].refresh)
            drift.assign(b->h_drift + b->drift_off[s], b->h_drift + b->drift_off[s] + e->W);
        const double wse = e->W > 1 ? std::sqrt(x[2] / (e->W - 1) / e->W) : 0.0;
        const SamplePass pass{steps, e->burn_in, (steps - e->burn_in) / e->batches, n_launch[s],
                              b->h_sys[s].refresh ? n_launch[s] : 0, o, (unsigned)x[0],
                              b->h_sys[s].refresh ? &drift : nullptr, (double)ms, sweep_ms, wse};
        vmc_sums sums{};
        std::vector<double> acc;
        rc = finish_sample(e, pass, &sums, acc);
        if (!rc) {
            b->last[s] = sums;
            rc = apply_sums(e, &sums, acc.data() + 9, acc.data() + 9 + e->EP, avg ? &avg[s] : nullptr, false);
        }
        b->theta_dirty[s] = 1;
        if (rc && !first_err) {
            first_err = rc;
            first_msg = "system " + std::to_string(s) + ": " + vmc_last_error();
        }
    }
    if (first_err) return bfail(first_err, first_msg);
    return VMC_OK;
}

int vmc_batch_last_sums(const vmc_batch *b, vmc_sums *out)
{
    if (!b || !out) return bfail(VMC_E_ARG, "null argument");
    std::copy(b->last.begin(), b->last.end(), out);
    return VMC_OK;
}

int vmc_batch_tuning(const vmc_batch *b, vmc_batch_candidate *out, int n)
{
    if (!b) return bfail(VMC_E_ARG, "null argument");
    const int m = (int)b->cands.size();
    for (int i = 0; i < m && i < n && out; ++i)
        out[i] = vmc_batch_candidate{b->cands[i].wpb, b->cands[i].per_item, b->cands[i].grid, b->cands[i].ns};
    return m;
}

}  // extern "C"

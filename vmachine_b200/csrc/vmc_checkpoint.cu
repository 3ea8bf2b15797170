// Checkpoint and resume.
//
// Parameter files in the reference's text format: Sampler::printParametersToFile
// (src/sampler.cpp:507-515) writes the E x P_max matrix through Eigen's default
// stream format, one row per line; FromFile (src/InitialWeights/fromfile.cpp:30-79)
// reads whitespace-separated numbers row by row.  Eigen 3's default format prints
// every coefficient right-aligned in one common width (the longest coefficient as
// printed with the stream's precision, 6 significant digits unless set), separated
// by one space, rows by a newline; the reference ends the file with endl.
//
// Walker state (no counterpart in the reference, which restarts from parameters
// only): a binary dump of everything a sampling pass reads, so a run resumed from it
// continues bit for bit: the records (positions and every derived array, in the
// engine's precision), FP64 running sums, Pade masks, Philox step counters, status
// words, the parameters, the optimiser's moments and step, the refresh cadence and
// the gamma history.
//
// Layout: "VMCSTATE" | u32 version | u32 header ints (n) | n x i32 header |
// u64 seed | f64 gamma_prev | sections, each u64 byte count + bytes, in the order
// theta, opt_m, opt_v, state, scal, mask, counter, status, and the learned MLP
// Jastrow dot's per-walker pair and one-body caches (empty for every other system).
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <iomanip>
#include <sstream>
#include <string>
#include <vector>

#include "vmc_engine.hpp"

using namespace vmc;

namespace {

int ck_fail(int code, const std::string &m) { return set_last_error(code, m.c_str()); }

#define CKCUDA(expr)                                                                         \
    do {                                                                                     \
        cudaError_t _e = (expr);                                                             \
        if (_e != cudaSuccess) return ck_fail(VMC_E_CUDA, std::string(#expr) + ": " + cudaGetErrorString(_e)); \
    } while (0)

std::string format_weights(const double *theta, int E, int P, int digits)
{
    auto coeff = [&](double v) {
        std::ostringstream s;
        s.precision(digits);
        s << v;
        return s.str();
    };
    size_t width = 0;
    for (int i = 0; i < E * P; ++i) width = std::max(width, coeff(theta[i]).size());
    std::ostringstream os;
    for (int i = 0; i < E; ++i) {
        if (i) os << '\n';
        for (int j = 0; j < P; ++j) {
            if (j) os << ' ';
            const std::string c = coeff(theta[(size_t)i * P + j]);
            os << std::string(width - c.size(), ' ') << c;
        }
    }
    os << '\n';
    return os.str();
}

const char MAGIC[8] = {'V', 'M', 'C', 'S', 'T', 'A', 'T', 'E'};
constexpr uint32_t STATE_VERSION = 2;

// header ints: what must match between the saving and the loading engine, then the
// run's progress
enum { H_N, H_DIM, H_W, H_PREC, H_GENERAL, H_E, H_PMAX, H_REC, H_ELEM, H_FLAGS, H_K, H_NACC, H_REFRESH,
       H_OPT_STEP, H_HAVE, H_COUNT };
constexpr int H_MATCH = H_NACC + 1;  // the first H_MATCH entries must agree
const char *H_NAMES[H_COUNT] = {"particles", "dimensions", "walkers", "precision", "path", "elements",
                                "parameters per element", "record length", "element bytes", "element flags",
                                "Hermite shells", "accumulators", "refresh interval", "optimiser step",
                                "walkers present"};

void header(const vmc_engine *e, int32_t *h)
{
    h[H_N] = e->N;
    h[H_DIM] = e->dim;
    h[H_W] = e->W;
    h[H_PREC] = e->precision;
    h[H_GENERAL] = e->general ? 1 : 0;
    h[H_E] = e->E;
    h[H_PMAX] = e->Pmax;
    h[H_REC] = e->L.rec;
    h[H_ELEM] = (int)e->elem_bytes;
    h[H_FLAGS] = e->flags;
    h[H_K] = e->K;
    h[H_NACC] = e->nacc_dev;
    h[H_REFRESH] = e->refresh_interval;
    h[H_OPT_STEP] = e->opt_step;
    h[H_HAVE] = e->have_walkers ? 1 : 0;
}

// floats of one walker's MLP Jastrow caches: (u, u', u'') of every ordered pair, then
// (chi, chi', chi'') of every particle
size_t mlp_cache_floats(const vmc_engine *e) { return (size_t)e->N * e->N * 3 + (size_t)e->N * 3; }

struct Section {
    void *dev;       // device buffer, or null
    void *host;      // host buffer, or null
    size_t bytes;
};

}  // namespace

namespace vmc {

// E x P_max parameters from a file in FromFile's format; "" or why not.
std::string read_weights_file(const std::string &path, int E, int P, std::vector<double> &theta)
{
    std::ifstream in(path);
    if (!in) return "cannot open weights file '" + path + "'";
    std::vector<std::vector<double>> rows;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ls(line);
        std::vector<double> r;
        double v;
        while (ls >> v) r.push_back(v);
        if (!r.empty()) rows.push_back(r);
    }
    if ((int)rows.size() != E)
        return "weights file has " + std::to_string(rows.size()) + " rows, expected " + std::to_string(E);
    theta.assign((size_t)E * P, 0.0);
    for (int i = 0; i < E; ++i) {
        if ((int)rows[i].size() != P)
            return "weights file row " + std::to_string(i) + " has " + std::to_string(rows[i].size()) +
                   " values, expected " + std::to_string(P);
        for (int j = 0; j < P; ++j) theta[(size_t)i * P + j] = rows[i][j];
    }
    return "";
}

int write_weights_file(const vmc_engine *e, const std::string &path, int digits)
{
    const std::string t = format_weights(e->theta.data(), e->E, e->Pmax, digits > 0 ? digits : 6);
    std::ofstream out(path);
    if (!out) return ck_fail(VMC_E_ARG, "cannot write '" + path + "'");
    out << t;
    return out ? VMC_OK : ck_fail(VMC_E_ARG, "cannot write '" + path + "'");
}

}  // namespace vmc

extern "C" {

long long vmc_format_weights(const double *theta, int n_elements, int p_max, int digits, char *buf, long long cap)
{
    if (!theta || n_elements < 1 || p_max < 1) return ck_fail(VMC_E_ARG, "bad parameter matrix");
    const std::string t = format_weights(theta, n_elements, p_max, digits > 0 ? digits : 6);
    if (buf && cap > 0) {
        const size_t n = std::min<size_t>(t.size(), (size_t)cap - 1);
        std::memcpy(buf, t.data(), n);
        buf[n] = 0;
    }
    return (long long)t.size();
}

int vmc_write_weights(const vmc_engine *e, const char *path, int digits)
{
    if (!e || !path) return ck_fail(VMC_E_ARG, "null argument");
    return write_weights_file(e, path, digits);
}

int vmc_read_weights(vmc_engine *e, const char *path)
{
    if (!e || !path) return ck_fail(VMC_E_ARG, "null argument");
    std::vector<double> th;
    const std::string why = read_weights_file(path, e->E, e->Pmax, th);
    if (!why.empty()) return ck_fail(VMC_E_CONFIG, why);
    return vmc_set_parameters(e, th.data(), e->E, e->Pmax);
}

int vmc_save_state(const vmc_engine *e, const char *path)
{
    if (!e || !path) return ck_fail(VMC_E_ARG, "null argument");
    CKCUDA(cudaSetDevice(e->device));
    CKCUDA(cudaStreamSynchronize(e->stream));
    const size_t W = e->W;
    const Section secs[] = {
        {nullptr, (void *)e->theta.data(), e->theta.size() * sizeof(double)},
        {nullptr, (void *)e->opt_m.data(), e->opt_m.size() * sizeof(double)},
        {nullptr, (void *)e->opt_v.data(), e->opt_v.size() * sizeof(double)},
        {e->d_state, nullptr, W * e->L.rec * e->elem_bytes},
        {e->d_scal, nullptr, W * NSCAL * sizeof(double)},
        {e->d_mask, nullptr, W * e->N * sizeof(unsigned long long)},
        {e->d_counter, nullptr, W * sizeof(unsigned long long)},
        {e->d_status, nullptr, W * sizeof(unsigned)},
        {e->d_mlp_cache, nullptr, e->d_mlp_cache ? W * mlp_cache_floats(e) * sizeof(float) : 0},
    };
    std::ofstream out(path, std::ios::binary);
    if (!out) return ck_fail(VMC_E_ARG, std::string("cannot write '") + path + "'");
    int32_t h[H_COUNT];
    header(e, h);
    const uint32_t ver = STATE_VERSION, nh = H_COUNT;
    const uint64_t seed = e->seed;
    const double gp = e->gamma_prev;
    out.write(MAGIC, 8);
    out.write((const char *)&ver, 4);
    out.write((const char *)&nh, 4);
    out.write((const char *)h, sizeof(h));
    out.write((const char *)&seed, 8);
    out.write((const char *)&gp, 8);
    std::vector<char> buf;
    for (const Section &s : secs) {
        const uint64_t n = s.bytes;
        out.write((const char *)&n, 8);
        if (s.dev) {
            buf.resize(s.bytes);
            CKCUDA(cudaMemcpy(buf.data(), s.dev, s.bytes, cudaMemcpyDeviceToHost));
            out.write(buf.data(), (std::streamsize)s.bytes);
        } else {
            out.write((const char *)s.host, (std::streamsize)s.bytes);
        }
    }
    return out ? VMC_OK : ck_fail(VMC_E_ARG, std::string("cannot write '") + path + "'");
}

int vmc_load_state(vmc_engine *e, const char *path)
{
    if (!e || !path) return ck_fail(VMC_E_ARG, "null argument");
    std::ifstream in(path, std::ios::binary);
    if (!in) return ck_fail(VMC_E_ARG, std::string("cannot open '") + path + "'");
    char magic[8];
    uint32_t ver = 0, nh = 0;
    in.read(magic, 8);
    in.read((char *)&ver, 4);
    in.read((char *)&nh, 4);
    if (!in || std::memcmp(magic, MAGIC, 8) != 0) return ck_fail(VMC_E_ARG, "not a walker-state file");
    if (ver != STATE_VERSION || nh != H_COUNT) return ck_fail(VMC_E_ARG, "walker-state file of another version");
    int32_t h[H_COUNT], mine[H_COUNT];
    uint64_t seed = 0;
    double gp = 0.0;
    in.read((char *)h, sizeof(h));
    in.read((char *)&seed, 8);
    in.read((char *)&gp, 8);
    header(e, mine);
    for (int i = 0; i < H_MATCH; ++i)
        if (h[i] != mine[i])
            return ck_fail(VMC_E_ARG, std::string("walker-state file is for another system: ") + H_NAMES[i] + " " +
                                          std::to_string(h[i]) + " != " + std::to_string(mine[i]));
    const size_t W = e->W;
    std::vector<double> th(e->theta.size()), m(e->opt_m.size()), v(e->opt_v.size());
    const Section secs[] = {
        {nullptr, th.data(), th.size() * sizeof(double)},
        {nullptr, m.data(), m.size() * sizeof(double)},
        {nullptr, v.data(), v.size() * sizeof(double)},
        {e->d_state, nullptr, W * e->L.rec * e->elem_bytes},
        {e->d_scal, nullptr, W * NSCAL * sizeof(double)},
        {e->d_mask, nullptr, W * e->N * sizeof(unsigned long long)},
        {e->d_counter, nullptr, W * sizeof(unsigned long long)},
        {e->d_status, nullptr, W * sizeof(unsigned)},
        {e->d_mlp_cache, nullptr, e->d_mlp_cache ? W * mlp_cache_floats(e) * sizeof(float) : 0},
    };
    std::vector<std::vector<char>> dev_bytes;
    for (const Section &s : secs) {
        uint64_t n = 0;
        in.read((char *)&n, 8);
        if (!in || n != s.bytes) return ck_fail(VMC_E_ARG, "walker-state file is truncated or inconsistent");
        if (s.dev) {
            dev_bytes.emplace_back(s.bytes);
            in.read(dev_bytes.back().data(), (std::streamsize)s.bytes);
        } else {
            in.read((char *)s.host, (std::streamsize)s.bytes);
        }
        if (!in) return ck_fail(VMC_E_ARG, "walker-state file is truncated");
    }
    // everything read: install it
    CKCUDA(cudaSetDevice(e->device));
    CKCUDA(cudaStreamSynchronize(e->stream));
    size_t di = 0;
    for (const Section &s : secs)
        if (s.dev) CKCUDA(cudaMemcpy(s.dev, dev_bytes[di++].data(), s.bytes, cudaMemcpyHostToDevice));
    e->opt_m = m;
    e->opt_v = v;
    e->opt_step = h[H_OPT_STEP];
    e->refresh_interval = h[H_REFRESH];
    e->seed = seed;
    e->have_walkers = h[H_HAVE] != 0;
    // the parameters without re-deriving the walkers (their derived arrays are restored)
    e->theta = th;
    e->gamma_prev = gp;
    return upload_parameters(e);
}

}  // extern "C"

// Oracle harness around the reference's own C++ classes (test infrastructure).
//
// Linked with the reference objects into oracle/_ref/libvmref.so.  It drives the
// reference through its public element interface, the same calls System makes:
//   - FixedPositions : InitialState   places walker at caller-given coordinates
//                                     (the reference's InitialState API,
//                                     src/InitialStates/initialstate.h:6-32)
//   - ReplayRNG : RandomNumberGenerator  returns a caller-given stream of numbers
//                                     in call order (src/RNG/rng.h:6-22), so the
//                                     reference and the GPU engine consume the
//                                     same uniforms and normals.
//   nextInt(n)        = floor(u * n)
//   nextDouble(lo,hi) = lo + (hi - lo) * u
//   nextGaussian(m,s) = m + s * z
// Private members of System/Sampler are reached by compiling this one file with
// the access keywords widened; the reference sources are unchanged.
#include <Eigen/Dense>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iostream>
#include <random>
#include <sstream>
#include <string>
#include <vector>
#include <unistd.h>

#define private public
#define protected public
#include "system.h"
#include "sampler.h"
#include "InitialStates/initialstate.h"
#include "Metropolis/metropolis.h"
#include "RNG/rng.h"
#include "WaveFunctions/wavefunction.h"
#include "Hamiltonians/hamiltonian.h"
#include "Interaction/interaction.h"
#include "Optimization/optimization.h"
#include "block/blocker.h"
#undef private
#undef protected

namespace {

class ReplayRNG : public RandomNumberGenerator
{
public:
    std::vector<double> stream;
    size_t pos = 0;
    bool exhausted = false;
    double next()
    {
        if (pos >= stream.size()) {
            exhausted = true;
            return 0.5;
        }
        return stream[pos++];
    }
    void setSeed(int) override {}
    int nextInt(int upperLimit) override { return int(std::floor(next() * upperLimit)); }
    double nextDouble(double lo, double hi) override { return lo + (hi - lo) * next(); }
    double nextGaussian(double mean, double sd) override { return mean + sd * next(); }
    std::string getLabel() override { return "replay"; }
    Eigen::MatrixXd randomUniformMatrix(Eigen::Index r, Eigen::Index c, double lo,
                                        double hi) override
    {
        Eigen::MatrixXd m(r, c);
        for (Eigen::Index i = 0; i < m.size(); i++) m.data()[i] = lo + (hi - lo) * next();
        return m;
    }
    Eigen::MatrixXd randomNormalMatrix(Eigen::Index r, Eigen::Index c, double mean,
                                       double sd) override
    {
        Eigen::MatrixXd m(r, c);
        for (Eigen::Index i = 0; i < m.size(); i++) m.data()[i] = mean + sd * next();
        return m;
    }
};

class FixedPositions : public InitialState
{
public:
    FixedPositions(System *s, const Eigen::VectorXd &p) : InitialState(s), fixed(p) {}
    Eigen::VectorXd fixed;
    std::string getLabel() override { return "fixed positions"; }
    void setupInitialState() override
    {
        m_numberOfDimensions = m_system->getNumberOfDimensions();
        m_numberOfParticles = m_system->getNumberOfParticles();
        m_degreesOfFreedom = m_system->getNumberOfFreeDimensions();
        m_positions = fixed;
        calculateDistanceMatrix();
        calculateRadialVector();
        for (auto &e : m_system->getWaveFunctionElements()) {
            e->initializeArrays(m_positions, m_radialVector, m_distanceMatrix);
            e->setArrays();
        }
    }
};

struct Handle
{
    System *sys = nullptr;
    FixedPositions *init = nullptr;
    ReplayRNG *rng = nullptr;
    std::string cfgPath;
    // snapshot for vmref_move / vmref_reset
    Eigen::VectorXd posOld;
    Eigen::MatrixXd distOld;
    Eigen::VectorXd radOld;
};

void syncFromInitialState(Handle *h)
{
    System *s = h->sys;
    s->m_positions = s->m_initialState->getParticles();
    s->m_distanceMatrix = s->m_initialState->getDistanceMatrix();
    s->m_radialVector = s->m_initialState->getRadialVector();
}

}  // namespace

extern "C" {

// Build a System from input.in text.  pos: D coordinates (particle-major).
// params: E x Pmax row-major (n_params entries) or NULL for the reference's own
// initial weights.  stream: the replayed random numbers.
void *vmref_create(const char *config_text, const double *pos, int n_pos, const double *params,
                   int n_params, const double *stream, long stream_len)
{
    Handle *h = new Handle();
    char tmpl[] = "/tmp/vmref_cfg_XXXXXX";
    int fd = mkstemp(tmpl);
    if (fd < 0) {
        delete h;
        return nullptr;
    }
    FILE *f = fdopen(fd, "w");
    fputs(config_text, f);
    fclose(f);
    h->cfgPath = tmpl;

    System *s = new System();
    h->sys = s;
    // main.cpp:8-10 defaults, applied before the configuration file is parsed
    s->setNumberOfParticles(2);
    s->setNumberOfDimensions(2);
    s->setEquilibrationFraction(0.001);

    Eigen::VectorXd p(n_pos);
    for (int i = 0; i < n_pos; i++) p(i) = pos[i];
    delete s->m_initialState;
    h->init = new FixedPositions(s, p);
    s->setInitialState(h->init);
    delete s->m_randomNumberGenerator;
    h->rng = new ReplayRNG();
    if (stream && stream_len > 0) h->rng->stream.assign(stream, stream + stream_len);
    s->setRandomNumberGenerator(h->rng);

    char arg0[] = "vmachine";
    std::vector<char> arg1(h->cfgPath.begin(), h->cfgPath.end());
    arg1.push_back('\0');
    char *argv[2] = {arg0, arg1.data()};
    s->initializeFromConfig(2, argv);
    s->initializeSystem();
    unlink(h->cfgPath.c_str());

    if (params) {
        int E = s->m_numberOfElements, P = s->m_maxParameters;
        if (n_params != E * P) {
            fprintf(stderr, "vmref_create: expected %d parameters, got %d\n", E * P, n_params);
            return nullptr;
        }
        Eigen::MatrixXd m(E, P);
        for (int i = 0; i < E; i++)
            for (int j = 0; j < P; j++) m(i, j) = params[i * P + j];
        s->m_parameters = m;
        s->updateAllParameters(m);
        s->m_initialState->setupInitialState();
        syncFromInitialState(h);
        s->m_metropolis->initialize();
    }
    // Initial weights of some element sets draw from the RNG (xavier.cpp:18,
    // randomuniform.cpp:18); rewind so the Metropolis steps consume the stream
    // from its first entry.
    h->rng->pos = 0;
    h->rng->exhausted = false;
    return h;
}

void vmref_destroy(void *hp)
{
    Handle *h = static_cast<Handle *>(hp);
    if (!h) return;
    // System's destructor frees the elements, the RNG and the initial state.
    delete h->sys;
    delete h;
}

// out: N, d, D, E, Pmax, numberOfBatches, stepsWOEqui, equilibrationSteps
int vmref_info(void *hp, int *out)
{
    Handle *h = static_cast<Handle *>(hp);
    System *s = h->sys;
    out[0] = s->m_numberOfParticles;
    out[1] = s->m_numberOfDimensions;
    out[2] = s->m_degreesOfFreedom;
    out[3] = s->m_numberOfElements;
    out[4] = s->m_maxParameters;
    out[5] = s->m_optimization->getNumberOfBatches();
    out[6] = s->m_stepsWOEqui;
    out[7] = s->m_equilibriationSteps;
    return 0;
}

int vmref_get_params(void *hp, double *out)
{
    Handle *h = static_cast<Handle *>(hp);
    const Eigen::MatrixXd &m = h->sys->m_parameters;
    for (int i = 0; i < m.rows(); i++)
        for (int j = 0; j < m.cols(); j++) out[i * m.cols() + j] = m(i, j);
    return 0;
}

int vmref_get_positions(void *hp, double *out)
{
    Handle *h = static_cast<Handle *>(hp);
    const Eigen::VectorXd &p = h->sys->m_positions;
    for (int i = 0; i < p.size(); i++) out[i] = p(i);
    return 0;
}

// Per element: gradient[D], Laplacian, parameter gradient[Pmax]; then
// energies = {T, V_ext, V_int} exactly as Sampler::sample forms them
// (src/sampler.cpp:66-70).
int vmref_eval(void *hp, double *grad, double *lap, double *pgrad, double *energies)
{
    Handle *h = static_cast<Handle *>(hp);
    System *s = h->sys;
    int D = s->m_degreesOfFreedom, P = s->m_maxParameters, e = 0;
    for (auto &el : s->m_waveFunctionElements) {
        for (int k = 0; k < D; k++) grad[e * D + k] = el->computeGradient(k);
        lap[e] = el->computeLaplacian();
        Eigen::VectorXd g = el->computeParameterGradient();
        for (int j = 0; j < P; j++) pgrad[e * P + j] = (j < g.size()) ? g(j) : 0.0;
        e++;
    }
    energies[0] = s->getKineticEnergy();
    energies[1] = s->m_hamiltonian->getExternalEnergy();
    energies[2] = s->m_interactionStyle->getInteractionEnergy();
    return 0;
}

// Move coordinate k to new_value the way Metropolis does (metropolis.cpp:21-39,
// then System::updateAllArrays) and report each element's evaluateRatio().
int vmref_move(void *hp, int k, double new_value, double *ratios)
{
    Handle *h = static_cast<Handle *>(hp);
    System *s = h->sys;
    int d = s->m_numberOfDimensions, N = s->m_numberOfParticles;
    h->posOld = s->m_positions;
    h->distOld = s->m_distanceMatrix;
    h->radOld = s->m_radialVector;
    Eigen::VectorXd pos = s->m_positions;
    pos(k) = new_value;
    int p = k / d;
    Eigen::MatrixXd dist = s->m_distanceMatrix;
    auto pd = [&](int i, int j) {
        double acc = 0;
        for (int a = 0; a < d; a++) {
            double diff = pos(d * i + a) - pos(d * j + a);
            acc += diff * diff;
        }
        return std::sqrt(acc);
    };
    for (int i = 0; i < p; i++) dist(i, p) = pd(p, i);
    for (int i = p + 1; i < N; i++) dist(p, i) = pd(p, i);
    Eigen::VectorXd rad = s->m_radialVector;
    if (rad.size() == N) {
        double acc = 0;
        for (int a = 0; a < d; a++) acc += pos(d * p + a) * pos(d * p + a);
        rad(p) = std::sqrt(acc);
    }
    s->m_positions = pos;
    s->m_distanceMatrix = dist;
    s->m_radialVector = rad;
    s->updateAllArrays(pos, rad, dist, k);
    int e = 0;
    for (auto &el : s->m_waveFunctionElements) ratios[e++] = el->evaluateRatio();
    return 0;
}

int vmref_reset(void *hp)
{
    Handle *h = static_cast<Handle *>(hp);
    System *s = h->sys;
    s->m_positions = h->posOld;
    s->m_distanceMatrix = h->distOld;
    s->m_radialVector = h->radOld;
    s->resetAllArrays();
    return 0;
}

// nsteps calls of Metropolis::acceptMove with the System copies refreshed as in
// System::runMetropolisCycles (system.cpp:149-153).  Records per step the
// accept flag, {T, V_ext, V_int}, and the parameter gradients (E x Pmax).
// Returns the number of random numbers consumed, or -1 if the stream ran out.
long vmref_steps(void *hp, int nsteps, unsigned char *accepted, double *energies, double *pgrads)
{
    Handle *h = static_cast<Handle *>(hp);
    System *s = h->sys;
    int E = s->m_numberOfElements, P = s->m_maxParameters;
    for (int i = 0; i < nsteps; i++) {
        bool acc = s->m_metropolis->acceptMove();
        s->m_positions = s->m_metropolis->updatePositions();
        s->m_distanceMatrix = s->m_metropolis->updateDistanceMatrix();
        s->m_radialVector = s->m_metropolis->updateRadialVector();
        if (accepted) accepted[i] = acc ? 1 : 0;
        if (energies) {
            energies[3 * i + 0] = s->getKineticEnergy();
            energies[3 * i + 1] = s->m_hamiltonian->getExternalEnergy();
            energies[3 * i + 2] = s->m_interactionStyle->getInteractionEnergy();
        }
        if (pgrads) {
            Eigen::MatrixXd g = s->getAllParameterGradients();
            for (int a = 0; a < E; a++)
                for (int b = 0; b < P; b++) pgrads[(size_t(i) * E + a) * P + b] = g(a, b);
        }
    }
    return h->rng->exhausted ? -1 : long(h->rng->pos);
}

// One optimisation iteration as System::runSimulation runs it
// (system.cpp:93-138) without files or terminal output:
// runMetropolisCycles, computeTotals, computeAverages, theta -= update.
// out: E, sigma_E, T, V_ext, V_int, acceptance ratio, then E*Pmax average
// gradients, E*Pmax average E*gradients, E*Pmax new parameters.
long vmref_iteration(void *hp, int iter, double *out)
{
    Handle *h = static_cast<Handle *>(hp);
    System *s = h->sys;
    Sampler *sm = s->m_sampler;
    s->m_iter = iter;
    sm->m_iter = iter;
    sm->setNumberOfSteps(s->m_stepsWOEqui, s->m_totalStepsWOEqui, s->m_totalStepsWEqui);
    s->runMetropolisCycles();
    sm->computeTotals();
    sm->computeAverages();
    s->m_parameters -= s->m_optimization->updateParameters();
    s->updateAllParameters(s->m_parameters);
    int E = s->m_numberOfElements, P = s->m_maxParameters;
    out[0] = sm->m_averageEnergy;
    out[1] = sm->m_stdError;
    out[2] = sm->m_averageKineticEnergy;
    out[3] = sm->m_averageExternalEnergy;
    out[4] = sm->m_averageInteractionEnergy;
    out[5] = double(sm->m_totalAcceptence) / sm->m_totalStepsWOEqui;
    size_t o = 6;
    for (int a = 0; a < E; a++)
        for (int b = 0; b < P; b++) out[o++] = sm->m_averageGradients(a, b);
    for (int a = 0; a < E; a++)
        for (int b = 0; b < P; b++) out[o++] = sm->m_averageGradientsE(a, b);
    for (int a = 0; a < E; a++)
        for (int b = 0; b < P; b++) out[o++] = s->m_parameters(a, b);
    return h->rng->exhausted ? -1 : long(h->rng->pos);
}

// System::runSimulation's iteration loop (system.cpp:91-137) without terminal or file
// output: adaptive steps from System::adaptiveSteps, the convergence check by
// System::checkingConvergence, set up as the API calls setConvergenceTools and
// setAdaptiveStepTools set them up (userinput.cpp:194-222) when check / adaptive are
// non-zero (the input.in keys alone leave the convergence window unsized).  Per
// iteration: the sampled steps (m_stepsWOEqui), the average energy, and 1 for the
// iteration that counts the densities and writes the instant energies.  Returns the
// iterations run, or -1 if the stream ran out.
long vmref_simulation(void *hp, int check, int n_energies, double tolerance, int adaptive, int range,
                      int additional, int additional_last, int *steps_out, double *energy_out, int *last_out)
{
    Handle *h = static_cast<Handle *>(hp);
    System *s = h->sys;
    Sampler *sm = s->m_sampler;
    if (check) s->setConvergenceTools(n_energies, tolerance);
    if (adaptive) s->setAdaptiveStepTools(range, additional, additional_last);
    s->m_numberOfNormalIterations = s->m_numberOfIterations - s->m_rangeOfAdaptiveSteps - 1;
    long n = 0;
    for (s->m_iter = 0; s->m_iter < s->m_numberOfIterations; s->m_iter++, n++) {
        if (s->m_applyAdaptiveSteps) {
            s->m_stepsWOEqui = s->m_initialStepsWOEqui * s->adaptiveSteps();
            s->m_stepsWEqui = s->m_stepsWOEqui + s->m_equilibriationSteps;
            s->m_totalStepsWOEqui = s->m_initialTotalStepsWOEqui * s->adaptiveSteps();
            s->m_totalStepsWEqui = s->m_totalStepsWOEqui + s->m_totalEquilibriationSteps;
        }
        sm->m_iter = s->m_iter;
        sm->setNumberOfSteps(s->m_stepsWOEqui, s->m_totalStepsWOEqui, s->m_totalStepsWEqui);
        steps_out[n] = s->m_stepsWOEqui;
        last_out[n] = s->m_iter == s->m_numberOfNormalIterations + s->m_rangeOfAdaptiveSteps ? 1 : 0;
        s->runMetropolisCycles();
        sm->computeTotals();
        sm->computeAverages();
        s->m_parameters -= s->m_optimization->updateParameters();
        energy_out[n] = sm->m_averageEnergy;
        if (s->m_checkConvergence) s->checkingConvergence();
        s->updateAllParameters(s->m_parameters);
    }
    return h->rng->exhausted ? -1 : n;
}

// nsteps Metropolis steps as vmref_steps, counting after every step the Sampler's
// electron densities from System's copies, as System::runMetropolisCycles does in the
// last iteration (system.cpp:157-160; Sampler::computeOneBodyDensity,
// computeOneBodyDensity2, computeTwoBodyDensity, sampler.cpp:639-692), on a grid of
// `bins` bins up to max_radius.  Outputs (each may be NULL, then not counted):
// radial[bins], spatial[bins][bins] (row = the y index), pair[bins][bins] (row = the
// bin of the lower-index particle).  Returns the random numbers consumed, or -1 if
// the stream ran out.
long vmref_densities(void *hp, int nsteps, int bins, double max_radius, long long *radial,
                     long long *spatial, long long *pair)
{
    Handle *h = static_cast<Handle *>(hp);
    System *s = h->sys;
    Sampler *sm = s->m_sampler;
    sm->m_computeOneBodyDensity = radial != nullptr;
    sm->m_computeOneBodyDensity2 = spatial != nullptr;
    sm->m_computeTwoBodyDensity = pair != nullptr;
    sm->m_numberOfBins = bins;
    sm->m_numberOfBinsHalf = bins / 2;
    sm->m_maxRadius = max_radius;
    sm->m_radialStep = max_radius / bins;
    sm->m_particlesPerBin = Eigen::VectorXi::Zero(bins);
    sm->m_densityGrid = Eigen::MatrixXi::Zero(bins, bins);
    sm->m_particlesPerBinPairwise = Eigen::MatrixXi::Zero(bins, bins);
    for (int i = 0; i < nsteps; i++) {
        s->m_metropolis->acceptMove();
        s->m_positions = s->m_metropolis->updatePositions();
        s->m_distanceMatrix = s->m_metropolis->updateDistanceMatrix();
        s->m_radialVector = s->m_metropolis->updateRadialVector();
        sm->computeOneBodyDensity(s->m_radialVector);
        sm->computeTwoBodyDensity(s->m_radialVector);
        sm->computeOneBodyDensity2(s->m_positions);
    }
    for (int r = 0; r < bins; r++) {
        if (radial) radial[r] = sm->m_particlesPerBin(r);
        for (int c = 0; c < bins; c++) {
            if (spatial) spatial[(size_t)r * bins + c] = sm->m_densityGrid(r, c);
            if (pair) pair[(size_t)r * bins + c] = sm->m_particlesPerBinPairwise(r, c);
        }
    }
    return h->rng->exhausted ? -1 : long(h->rng->pos);
}

// Blocker on a series of length 2^k (include/block/blocker.cpp:15-33):
// out = {mean, stdErr}.
int vmref_blocking(const double *x, long n, double *out)
{
    std::vector<double> v(x, x + n);
    Blocker b(v);
    out[0] = b.mean;
    out[1] = b.stdErr;
    return 0;
}

// The reference's parameter file text for an E x P row-major matrix
// (Sampler::printParametersToFile, sampler.cpp:507-515: the matrix through Eigen's
// default stream format, then endl).  Returns the length; writes at most cap - 1
// characters and a terminating zero.
long vmref_format_weights(const double *theta, int E, int P, char *buf, long cap)
{
    Eigen::MatrixXd m(E, P);
    for (int i = 0; i < E; i++)
        for (int j = 0; j < P; j++) m(i, j) = theta[i * P + j];
    std::ostringstream os;
    os << m << std::endl;
    const std::string t = os.str();
    if (cap > 0) {
        const long n = std::min<long>((long)t.size(), cap - 1);
        std::memcpy(buf, t.data(), n);
        buf[n] = 0;
    }
    return (long)t.size();
}

// System's settings after parsing and set-up, as doubles in this order: particles,
// dimensions, omega, sigma, Z, hidden units, learning rate, iterations, equilibration
// fraction, total steps without burn-in, step length, sorting, max radius, bins,
// tolerance, energies kept by the convergence check, range of adaptive steps,
// additional steps, additional steps in the last iteration, checkpoint frequency, and
// the convergence-check, adaptive-steps and three density switches.  Returns 25.
int vmref_settings(void *hp, double *out)
{
    const System *s = static_cast<Handle *>(hp)->sys;
    const double v[] = {double(s->m_numberOfParticles), double(s->m_numberOfDimensions), s->m_omega,
                        s->m_sigma, double(s->m_Z), double(s->m_numberOfHiddenUnits), s->m_eta,
                        double(s->m_numberOfIterations), s->m_equilibrationFraction,
                        double(s->m_initialTotalStepsWOEqui), s->m_stepLength, double(s->m_sorting),
                        s->m_maxRadius, double(s->m_numberOfBins), s->m_tolerance,
                        double(s->m_numberOfEnergies), double(s->m_rangeOfAdaptiveSteps),
                        double(s->m_additionalSteps), double(s->m_additionalStepsLastIter),
                        double(s->m_checkpointFreq), double(s->m_checkConvergence),
                        double(s->m_applyAdaptiveSteps), double(s->m_computeOneBodyDensity),
                        double(s->m_computeOneBodyDensity2), double(s->m_computeTwoBodyDensity)};
    const int n = int(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < n; i++) out[i] = v[i];
    return n;
}

// System's trial wave-function label (System::collectAllLabels, parser.cpp:396-520),
// the name Automatize reads to choose the initial weights.  Writes it NUL-terminated
// into buf and returns its length, or -1 if cap is too small.
long vmref_trial_label(void *hp, char *buf, long cap)
{
    const std::string t = static_cast<Handle *>(hp)->sys->getTrialWaveFunction();
    if ((long)t.size() + 1 > cap) return -1;
    std::memcpy(buf, t.c_str(), t.size() + 1);
    return (long)t.size();
}

}  // extern "C"

// Reference-side adapter of the B200 engine (see b200engine.h).
#include "b200engine.h"

#include <cmath>
#include <cstdio>

#include "InitialStates/initialstate.h"
#include "RNG/rng.h"
#include "system.h"

// ------------------------------------------------------------------ B200Engine

B200Engine::B200Engine(const std::string &inputText, const vmc_options *opt)
{
    check(vmc_create(inputText.c_str(), opt, &m_e));
    check(vmc_get_info(m_e, &m_info));
}

B200Engine::~B200Engine() { vmc_destroy(m_e); }

void B200Engine::check(int rc) const
{
    if (rc != VMC_OK) throw B200Error{rc, vmc_last_error()};
}

void B200Engine::initializeWalkers(uint64_t seed) { check(vmc_init_walkers(m_e, nullptr, seed)); }

void B200Engine::initializeWalkers(const Eigen::MatrixXd &positions, uint64_t seed)
{
    if (positions.rows() != m_info.n_walkers || positions.cols() != m_info.n_coords)
        throw B200Error{VMC_E_ARG, "positions must be numberOfWalkers x D"};
    // the C ABI takes walker-major rows (particle-major coordinates, as System::m_positions)
    const Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor> rows = positions;
    check(vmc_init_walkers(m_e, rows.data(), seed));
}

vmc_averages B200Engine::runIteration(int iteration)
{
    vmc_averages a{};
    check(vmc_run_iteration(m_e, iteration, &a));
    return a;
}

vmc_sums B200Engine::sample(int iteration, Eigen::MatrixXd &gradSum, Eigen::MatrixXd &eGradSum)
{
    const int E = m_info.n_elements, P = m_info.p_max;
    Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor> g(E, P), ge(E, P);
    vmc_sums s{};
    check(vmc_sample(m_e, iteration, m_info.steps_per_walker + m_info.burn_in, m_info.burn_in, &s, g.data(),
                     ge.data()));
    gradSum = g;
    eGradSum = ge;
    return s;
}

vmc_averages B200Engine::applySums(const vmc_sums &sums, const Eigen::MatrixXd &gradSum,
                                   const Eigen::MatrixXd &eGradSum)
{
    const Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor> g = gradSum, ge = eGradSum;
    vmc_averages a{};
    check(vmc_apply_sums(m_e, &sums, g.data(), ge.data(), &a));
    return a;
}

Eigen::MatrixXd B200Engine::parameters() const
{
    Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor> t(m_info.n_elements, m_info.p_max);
    check(vmc_get_parameters(m_e, t.data(), m_info.n_elements, m_info.p_max));
    return t;
}

void B200Engine::setParameters(const Eigen::MatrixXd &theta)
{
    if (theta.rows() != m_info.n_elements || theta.cols() != m_info.p_max)
        throw B200Error{VMC_E_ARG, "parameters must be numberOfElements x maxParameters"};
    const Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor> t = theta;
    check(vmc_set_parameters(m_e, t.data(), m_info.n_elements, m_info.p_max));
}

Eigen::MatrixXd B200Engine::positions() const
{
    Eigen::Matrix<double, Eigen::Dynamic, Eigen::Dynamic, Eigen::RowMajor> x(m_info.n_walkers, m_info.n_coords);
    check(vmc_get_positions(m_e, x.data()));
    return x;
}

// ------------------------------------------------------------------ B200Optimization

B200Optimization::B200Optimization(System *system, B200Engine *engine)
    : Optimization(system), m_engine(engine)
{}

int B200Optimization::getNumberOfBatches() { return m_engine->info().batches; }

vmc_averages B200Optimization::iterate(int iteration)
{
    const Eigen::MatrixXd before = m_engine->parameters();
    const vmc_averages a = m_engine->runIteration(iteration);
    m_step = before - m_engine->parameters();
    m_have_step = true;
    m_iteration = iteration + 1;
    return a;
}

Eigen::MatrixXd B200Optimization::updateParameters()
{
    if (!m_have_step) iterate(m_iteration);
    m_have_step = false;
    return m_step;
}

// ------------------------------------------------------------------ B200Metropolis

B200Metropolis::B200Metropolis(System *system, const std::string &inputText, int device)
    : Metropolis(system), m_text(inputText), m_device(device)
{}

B200Metropolis::~B200Metropolis() { delete m_engine; }

void B200Metropolis::initialize()
{
    // the same fields ImportanceSampling::initialize and BruteForce::initialize set
    // (importancesampling.cpp:11-32, bruteforce.cpp:11-24)
    m_numberOfDimensions = m_system->getNumberOfDimensions();
    m_numberOfParticles = m_system->getNumberOfParticles();
    m_degreesOfFreedom = m_system->getNumberOfFreeDimensions();
    m_stepLength = m_system->getStepLength();
    m_positions = m_system->getInitialState()->getParticles();
    m_radialVector = m_system->getInitialState()->getRadialVector();
    m_distanceMatrix = m_system->getInitialState()->getDistanceMatrix();
    m_system->setGlobalArraysToCalculate();
    m_calculateDistanceMatrix = m_system->getCalculateDistanceMatrix();
    m_calculateRadialVector = m_system->getCalculateRadialVector();
    m_RNG = m_system->getRandomNumberGenerator();
    m_importance = m_text.find("bruteForce") == std::string::npos;

    // one walker in FP64 with the reference's quirks: System's walker, moved on the GPU
    vmc_options o{};
    o.device = m_device;
    o.precision = VMC_PRECISION_FP64;
    o.num_walkers = 1;
    o.walkers_per_block = 0;
    o.refresh_interval = -1;
    o.compat = 1;
    delete m_engine;
    m_engine = new B200Engine(m_text, &o);
    m_theta = m_system->getWeights();
    m_engine->setParameters(m_theta);
    m_engine->initializeWalkers(Eigen::MatrixXd(m_positions.transpose()));
}

bool B200Metropolis::acceptMove()
{
    // parameters are updated between iterations (System::updateAllParameters)
    const Eigen::MatrixXd theta = m_system->getWeights();
    if (theta.rows() != m_theta.rows() || theta.cols() != m_theta.cols() || theta != m_theta) {
        m_theta = theta;
        m_engine->setParameters(m_theta);
    }
    // the reference's draws in its order; the engine reads nextInt as floor(u D)
    const int i = m_RNG->nextInt(m_degreesOfFreedom);
    const double z = m_importance ? m_RNG->nextGaussian(0, 1) : m_RNG->nextDouble();
    const double u = m_RNG->nextDouble();
    const double stream[3] = {(i + 0.5) / m_degreesOfFreedom, z, u};
    uint8_t accepted = 0;
    const int rc = vmc_replay(m_engine->handle(), stream, 1, &accepted, nullptr);
    if (rc != VMC_OK) throw B200Error{rc, vmc_last_error()};
    if (!accepted) return false;
    // the walker where the engine put it; System's elements follow (updateAllArrays),
    // as after an accepted move of the reference's own Metropolis
    m_positions(i) = m_engine->positions()(0, i);
    const int particle = i / m_numberOfDimensions;
    if (m_calculateDistanceMatrix) Metropolis::calculateDistanceMatrixCross(particle);
    if (m_calculateRadialVector) Metropolis::calculateRadialVectorElement(particle);
    m_system->updateAllArrays(m_positions, m_radialVector, m_distanceMatrix, i);
    return true;
}

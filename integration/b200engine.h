// The B200 engine inside a VMaChine build: the reference-side adapter over the C ABI
// (include/vmc_b200.h).  Compiled with VMaChine's own headers (src/, Eigen) and linked
// against libvmc_b200.so; integration/Makefile builds it next to the reference sources.
//
//   B200Engine        the walker population on the GPU behind Eigen types: one call per
//                     iteration of System::runSimulation's loop (src/system.cpp:93-138):
//                     runMetropolisCycles + Sampler::sample + computeTotals (vmc_sample),
//                     computeAverages + the optimiser step + updateAllParameters
//                     (vmc_apply_sums).
//   B200Optimization  an Optimization (src/Optimization/optimization.h) whose
//                     updateParameters() returns the step the engine took, so the
//                     reference's `m_parameters -= m_optimization->updateParameters()`
//                     (system.cpp:114) keeps System's parameters equal to the engine's.
//   B200Metropolis    a Metropolis (src/Metropolis/metropolis.h) that moves System's own
//                     walker on the GPU: each acceptMove() draws the reference's random
//                     numbers from System's generator in the reference's order (nextInt,
//                     nextGaussian or nextDouble, nextDouble; importancesampling.cpp:49-81,
//                     bruteforce.cpp:26-52), lets a one-walker engine decide the move on
//                     them (vmc_replay), and on acceptance updates System's element arrays
//                     (System::updateAllArrays) so the reference's Sampler sees the walker
//                     where the engine put it.  One launch per move: it exists to run
//                     System::runSimulation unchanged around the engine, the population
//                     path above is the fast one.
#pragma once
#include <Eigen/Dense>
#include <string>
#include <vector>

#include "Metropolis/metropolis.h"
#include "Optimization/optimization.h"
#include "vmc_b200.h"

// Thrown on any engine error (the C ABI's negative return codes).
struct B200Error {
    int code;
    std::string message;
};

class B200Engine
{
public:
    // input.in text in the reference's key schema (System::parser, parser.cpp:25-333)
    // plus the engine's keys (numWalkers, precision, ...); opt may be null.
    explicit B200Engine(const std::string &inputText, const vmc_options *opt = nullptr);
    ~B200Engine();
    B200Engine(const B200Engine &) = delete;
    B200Engine &operator=(const B200Engine &) = delete;

    // InitialState::setupInitialState + Metropolis::initialize for every walker: the
    // configured initial state from per-walker Philox streams, or the given positions
    // (numberOfWalkers rows of D coordinates)
    void initializeWalkers(uint64_t seed);
    void initializeWalkers(const Eigen::MatrixXd &positions, uint64_t seed = 0);

    // one pass of System::runSimulation's loop: returns the averages of the pass
    // (Sampler::computeAverages) after the optimiser step has been applied
    vmc_averages runIteration(int iteration);
    // the same in two halves: the sampling pass (runMetropolisCycles, Sampler::sample,
    // computeTotals), then averages, optimiser step and parameter update from totals
    // that may come from several engines (MPI_Reduce in the reference)
    vmc_sums sample(int iteration, Eigen::MatrixXd &gradSum, Eigen::MatrixXd &eGradSum);
    vmc_averages applySums(const vmc_sums &sums, const Eigen::MatrixXd &gradSum, const Eigen::MatrixXd &eGradSum);

    Eigen::MatrixXd parameters() const;                // System::m_parameters (E x P_max)
    void setParameters(const Eigen::MatrixXd &theta);  // System::updateAllParameters
    Eigen::MatrixXd positions() const;                 // W x D

    const vmc_info &info() const { return m_info; }
    vmc_engine *handle() { return m_e; }

private:
    void check(int rc) const;
    vmc_engine *m_e = nullptr;
    vmc_info m_info{};
};

class B200Optimization : public Optimization
{
public:
    // engine: the population that samples the iterations (owned by the caller)
    B200Optimization(class System *system, B200Engine *engine);
    int getNumberOfBatches() override;
    std::string getLabel() override { return "B200 engine optimiser"; }
    void initialize() override {}
    // the step of the iteration the engine sampled last: parameters before minus after
    // (the engine has applied it); the first call samples an iteration if none was
    Eigen::MatrixXd updateParameters() override;
    // sample and step one iteration; updateParameters() then reports its step
    vmc_averages iterate(int iteration);

private:
    B200Engine *m_engine;
    Eigen::MatrixXd m_step;
    bool m_have_step = false;
    int m_iteration = 0;
};

class B200Metropolis : public Metropolis
{
public:
    // inputText: the input.in the System was configured from (the engine parses its own
    // copy as a one-walker FP64 engine with the same elements and sampler)
    B200Metropolis(class System *system, const std::string &inputText, int device = 0);
    ~B200Metropolis() override;
    std::string getLabel() override { return m_label; }
    void initialize() override;
    bool acceptMove() override;

private:
    std::string m_text, m_label = "Metropolis on the B200 engine";
    int m_device;
    bool m_importance = true;
    B200Engine *m_engine = nullptr;
    Eigen::MatrixXd m_theta;  // the parameters last pushed to the engine
};

// input.in parsing with the reference's semantics (src/parser.cpp:25-333,
// src/userinput.cpp:60-81, defaults from src/system.h:266-310 and src/main.cpp:8-10).
#pragma once
#include <string>
#include <vector>

namespace vmc {

enum Element { E_GAUSSIAN = 0, E_SLATER = 1, E_PADE = 2, E_SIMPLEJASTROW = 3,
               E_RBMGAUSSIAN = 4, E_RBMPRODUCT = 5, E_HYDROGENLIKE = 6,
               E_MLP = 7,  // learned MLP Jastrow (no counterpart in the reference)
               E_OTHER = 99 };

// MLP Jastrow shape: pair network 2 -> 64 -> 64 -> 1, one-body network 1 -> 32 -> 32 -> 1
constexpr int MLP_H = 64, MLP_G = 32;
constexpr int MLP_PARAMS = MLP_H * 2 + MLP_H + MLP_H * MLP_H + MLP_H + MLP_H + 1 +
                           MLP_G + MLP_G + MLP_G * MLP_G + MLP_G + MLP_G + 1;  // 5570

struct Config {
    // system
    int N = 2, dim = 2;          // main.cpp:8-9
    double omega = 1.0;
    double sigma = 1.0;          // RBM width; `omega:` sets 1/sqrt(omega) (parser.cpp:57-60)
    int Z = 2;                   // `numParticles:` sets Z = N, `atomicNumber:` overrides
    int hidden = 2;              // `numParticles:` sets hidden = N (parser.cpp:52-54)
    std::string hamiltonian;     // harmonicOscillator | atomicNucleus
    bool coulomb = false;        // interactionStyle
    std::string basis = "none";  // hermite | hydrogenOrbital
    std::vector<int> elements;   // Element codes, configuration order
    std::string trial_label;     // collectAllLabels result ("VMC", "RBM", ...)
    // simulation
    double eta = 0.1;            // learningRate (system.h:297)
    int iterations = 100;
    double eq_fraction = 0.001;  // main.cpp:10
    long long num_steps = 1LL << 19;  // system.h:276
    double step_length = 0.05;   // system.h:296; `omega:` sets 0.1/sqrt(omega)
    bool sorting = true;
    std::string sampling = "importanceSampling";
    std::string optimization = "adam";
    double opt_gamma = 0.0, opt_power = 0.0;  // gd/sgd momentum and monotonic power
    std::string initial_weights = "automatize";
    double weights_factor = 1.0;
    std::string weights_file;
    std::string initial_state = "randomNormal";
    bool have_seed = false;
    long long seed = 0;
    // output/driver keys (accepted, mostly informational)
    double max_radius = 5.0, total_spin = 0.0, tolerance = 1e-7;
    int checkpoint_freq = 100, n_energies = 5, range_adaptive = 10, add_steps = 4,
        add_steps_last = 8, n_bins = 1000;
    bool check_convergence = false, adaptive_steps = false, ob_density = false,
         ob_density2 = false, tb_density = false, print_energy = false, print_params = false,
         do_resampling = false;
    std::string path;
    // engine keys (new)
    int walkers = 1;
    int walker_offset = 0;       // this engine's first walker in a sharded population (random streams)
    // importance sampling, corrected mode: drift limiter constant a (0: off), the drift
    // v = d ln Psi / dx scaled to 2 v / (1 + sqrt(1 + 2 a dt v^2)) in the proposal and
    // in the Green's ratio (Umrigar, Nightingale and Runge, J. Chem. Phys. 99, 2865 (1993))
    double drift_limit = 0.0;
    int precision = 0;           // 0 fp64, 1 mixed
    int refresh_interval = -1;   // -1 auto
    int compat = 1;              // 1 reference quirks, 0 corrected
    bool mlp_tc = true;          // MLP Jastrow second layer on the tensor cores (mlpTensorCores)
    int walkers_per_block = 0;   // 0 auto
    int walkers_per_warp = 0;    // at most this many walkers per warp: 0 auto (4 for dots of N <= 6, 2 for N = 12 to 30), 1, 2, 4
    int sweep_form = 0;          // production dot sweep: 0 auto (owner for one walker per warp), 1 staged, 2 owner
};

// Returns empty string on success, else an error message.
std::string parse_config(const std::string &text, Config &cfg);

// Number of parameters per element (the reference's getNumberOfParameters after
// setConstants: slaterdeterminant.h:42, simplejastrow.cpp:15, rbmgaussian.cpp:12,
// rbmproduct.cpp:101, others 1).
int element_parameters(const Config &cfg, int element);

}  // namespace vmc

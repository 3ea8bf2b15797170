// input.in parser.  Same key schema and side effects as the reference
// (src/parser.cpp:25-333): `#` comments at column 0, `key: value` lines, unknown
// keys rejected, `omega:` resets stepLength and the RBM width, `numParticles:`
// resets the hidden-node count and Z.  Errors are returned, not aborted on.
#include "vmc_config.hpp"

#include <algorithm>
#include <cmath>
#include <sstream>

namespace vmc {

namespace {

std::string trim(const std::string &s)
{
    const char *ws = " \t\n\r\f\v";
    const size_t b = s.find_first_not_of(ws);
    if (b == std::string::npos) return "";
    const size_t e = s.find_last_not_of(ws);
    return s.substr(b, e - b + 1);
}

std::vector<std::string> split(const std::string &s)
{
    std::istringstream iss(s);
    std::vector<std::string> out;
    std::string t;
    while (iss >> t) out.push_back(t);
    return out;
}

bool parse_bool(const std::string &s, bool &out)
{
    if (s == "true") { out = true; return true; }
    if (s == "false") { out = false; return true; }
    return false;
}

const char *element_label(int e)
{
    switch (e) {
    case E_GAUSSIAN: return "Gaussian";
    case E_SLATER: return "Slater determinant";
    case E_PADE: return "Pad\xc3\xa9-Jastrow";
    case E_SIMPLEJASTROW: return "simple Jastrow";
    case E_RBMGAUSSIAN: return "RBM-Gaussian";
    case E_RBMPRODUCT: return "RBM-product";
    case E_HYDROGENLIKE: return "hydrogenlike";
    case E_MLP: return "MLP-Jastrow";
    default: return "other";
    }
}

// System::searchShortning (parser.cpp:340-390) as a rule on the labels: the
// concatenated string "_l1_l2..." takes the short name when it holds as many labels as
// `labels` (at most four), each of them one of `labels`, and they are not all the same
// one (a one-label list matches itself).  Repeats are allowed otherwise: the
// reference's loops accept e.g. "_Gaussian_Gaussian_Pade-Jastrow" for three labels.
void shortening(const std::vector<std::string> &labels, const std::string &name, std::string &all)
{
    if (all.empty() || all[0] != '_' || labels.size() > 4) return;
    std::vector<std::string> parts;
    for (size_t a = 1; a <= all.size();) {
        size_t b = all.find('_', a);
        if (b == std::string::npos) b = all.size();
        parts.push_back(all.substr(a, b - a));
        a = b + 1;
    }
    if (parts.size() != labels.size()) return;
    bool uniform = true;
    for (const std::string &p : parts) {
        if (std::find(labels.begin(), labels.end(), p) == labels.end()) return;
        uniform = uniform && p == parts[0];
    }
    if (labels.size() == 1 || !uniform) all = name;
}

// System::collectAllLabels (parser.cpp:396-520)
std::string trial_label(const std::vector<int> &elements)
{
    std::string all;
    for (int e : elements) all += std::string("_") + element_label(e);
    const std::string G = "Gaussian", P = "Pad\xc3\xa9-Jastrow", S = "Slater determinant",
                      RG = "RBM-Gaussian", RP = "RBM-product", SJ = "simple Jastrow",
                      H = "hydrogenlike";
    shortening({G}, "VMC", all);
    shortening({G, P}, "VMC", all);
    shortening({G, P, S}, "VMC", all);
    shortening({RG, RP}, "RBM", all);
    shortening({RG, RP, S}, "RBM", all);
    shortening({RG, RP, P}, "RBMPJ", all);
    shortening({RG, RP, P, S}, "RBMPJ", all);
    shortening({RG, RP, SJ}, "RBMSJ", all);
    shortening({RG, RP, SJ, S}, "RBMSJ", all);
    shortening({H}, "VMC", all);
    shortening({S}, "VMC", all);
    shortening({H, P}, "VMC", all);
    shortening({S, P}, "VMC", all);
    shortening({S, G}, "VMC", all);
    shortening({S, G, SJ}, "SSJ", all);
    shortening({G, SJ}, "SSJ", all);
    return all;
}

}  // namespace

int element_parameters(const Config &cfg, int e)
{
    const int D = cfg.N * cfg.dim;
    switch (e) {
    case E_SLATER: return 0;
    case E_SIMPLEJASTROW: return cfg.N * cfg.N;
    case E_RBMGAUSSIAN: return D;
    case E_RBMPRODUCT: return cfg.hidden * D + cfg.hidden;
    case E_MLP: return MLP_PARAMS;
    default: return 1;
    }
}

std::string parse_config(const std::string &text, Config &c)
{
    std::istringstream in(text);
    std::string line;
    int lineno = 0;
    while (std::getline(in, line)) {
        ++lineno;
        if (line.empty() || line.rfind("#", 0) == 0) continue;
        const size_t colon = line.find(':');
        if (colon == std::string::npos) {
            // the reference's getline(is_line, key, ':') accepts a line without a
            // colon as a key with no value, which it then skips
            if (trim(line).empty()) continue;
            continue;
        }
        const std::string key = trim(line.substr(0, colon));
        const std::vector<std::string> v = split(line.substr(colon + 1));
        if (v.empty()) continue;  // key with no value: the reference reads nothing
        const std::string &v0 = v[0];
        auto err = [&](const std::string &m) {
            return "input.in line " + std::to_string(lineno) + ": " + m;
        };
        try {
            bool bv = false;
            if (key == "numParticles") {
                c.N = std::stoi(v0);
                c.hidden = c.N;
                c.Z = c.N;
            } else if (key == "numDimensions") {
                c.dim = std::stoi(v0);
            } else if (key == "omega") {
                c.omega = std::stod(v0);
                c.step_length = 0.1 / std::sqrt(c.omega);
                c.sigma = 1.0 / std::sqrt(c.omega);
            } else if (key == "atomicNumber") {
                c.Z = std::stoi(v0);
            } else if (key == "learningRate") {
                c.eta = std::stod(v0);
            } else if (key == "maxRadius") {
                c.max_radius = std::stod(v0);
            } else if (key == "numIterations") {
                c.iterations = std::stoi(v0);
            } else if (key == "equilibration") {
                c.eq_fraction = std::stod(v0);
            } else if (key == "numSteps") {
                c.num_steps = std::stoll(v0);
            } else if (key == "numHiddenNodes") {
                c.hidden = std::stoi(v0);
            } else if (key == "sorting") {
                if (parse_bool(v0, bv)) c.sorting = bv;
            } else if (key == "totalSpin") {
                c.total_spin = std::stod(v0);
            } else if (key == "stepLength") {
                c.step_length = std::stod(v0);
            } else if (key == "checkpointFreq") {
                c.checkpoint_freq = (int)std::stod(v0);
            } else if (key == "checkConvergence") {
                if (parse_bool(v0, bv)) c.check_convergence = bv;
            } else if (key == "applyAdaptiveSteps") {
                if (parse_bool(v0, bv)) c.adaptive_steps = bv;
            } else if (key == "computeOneBodyDensity") {
                if (parse_bool(v0, bv)) c.ob_density = bv;
            } else if (key == "computeOneBodyDensity2") {
                if (parse_bool(v0, bv)) c.ob_density2 = bv;
            } else if (key == "computeTwoBodyDensity") {
                if (parse_bool(v0, bv)) c.tb_density = bv;
            } else if (key == "printEnergyToFile") {
                if (parse_bool(v0, bv)) c.print_energy = bv;
            } else if (key == "printParametersToFile") {
                if (parse_bool(v0, bv)) c.print_params = bv;
            } else if (key == "doResampling") {
                if (parse_bool(v0, bv)) c.do_resampling = bv;
            } else if (key == "path") {
                c.path = v0;
            } else if (key == "numberOfEnergies") {
                c.n_energies = std::stoi(v0);
            } else if (key == "tolerance") {
                c.tolerance = std::stod(v0);
            } else if (key == "rangeOfAdaptiveSteps") {
                c.range_adaptive = std::stoi(v0);
            } else if (key == "additionalSteps") {
                c.add_steps = std::stoi(v0);
            } else if (key == "additionalStepsLastIter") {
                c.add_steps_last = std::stoi(v0);
            } else if (key == "numberOfBins") {
                c.n_bins = std::stoi(v0);
            } else if (key == "basis") {
                if (v0 != "hermite" && v0 != "hydrogenOrbital")
                    return err("Basis '" + v0 + "' is not implemented!");
                c.basis = v0;
            } else if (key == "hamiltonian") {
                if (v0 != "harmonicOscillator" && v0 != "atomicNucleus" && v0 != "doubleWell" &&
                    v0 != "ellipticalHarmonicOscillator")
                    return err("The Hamiltonian '" + v0 + "' does not exist!");
                c.hamiltonian = v0;
            } else if (key == "optimization") {
                if (v0 == "adam") {
                    c.optimization = "adam";
                } else if (v0 == "gd" || v0 == "sgd") {
                    c.optimization = v0;
                    c.opt_gamma = v.size() >= 3 ? std::stod(v[1]) : 0.0;
                    c.opt_power = v.size() >= 3 ? std::stod(v[2]) : 0.0;
                } else {
                    return err("Optimization method '" + v0 + "' does not exist!");
                }
            } else if (key == "initialWeights") {
                if (v0 == "automatize") {
                    c.initial_weights = v0;
                } else if (v0 == "randomuniform") {
                    c.initial_weights = v0;
                    c.weights_factor = v.size() >= 2 ? std::stod(v[1]) : 1.0;
                } else if (v0 == "constant") {
                    c.initial_weights = v0;
                    c.weights_factor = v.size() >= 2 ? std::stod(v[1]) : 1.0;
                } else if (v0 == "fromfile") {
                    c.initial_weights = v0;
                    c.weights_file = v.size() >= 2 ? v[1] : "weights.dat";
                } else {
                    return err("Initial parameter configuration '" + v0 + "' does not exist!");
                }
            } else if (key == "initialState") {
                if (v0 != "randomNormal" && v0 != "randomUniform")
                    return err("Initial state configuration '" + v0 + "' does not exist!");
                c.initial_state = v0;
            } else if (key == "sampling") {
                if (v0 != "importanceSampling" && v0 != "bruteForce")
                    return err("Sampling method '" + v0 + "' does not exist!");
                c.sampling = v0;
            } else if (key == "waveFunction") {
                // parser.cpp:223-262; for VMC the Gaussian pushed first is dropped when
                // the element list is replaced, leaving Slater x Pade.
                c.elements.clear();
                if (v0 == "VMC") c.elements = {E_SLATER, E_PADE};
                else if (v0 == "RBM") c.elements = {E_SLATER, E_RBMGAUSSIAN, E_RBMPRODUCT};
                else if (v0 == "RBMPJ") c.elements = {E_SLATER, E_RBMGAUSSIAN, E_RBMPRODUCT, E_PADE};
                else if (v0 == "RBMSJ") c.elements = {E_SLATER, E_RBMGAUSSIAN, E_RBMPRODUCT, E_SIMPLEJASTROW};
                else if (v0 == "PRBM") c.elements = {E_SLATER, E_RBMGAUSSIAN, E_RBMPRODUCT, E_OTHER};
                else return err("Wave function '" + v0 + "' does not exist!");
            } else if (key == "waveFunctionElement") {
                if (v0 == "gaussian") c.elements.push_back(E_GAUSSIAN);
                else if (v0 == "slaterDeterminant") c.elements.push_back(E_SLATER);
                else if (v0 == "padeJastrow") c.elements.push_back(E_PADE);
                else if (v0 == "simpleJastrow") c.elements.push_back(E_SIMPLEJASTROW);
                else if (v0 == "RBMGaussian") c.elements.push_back(E_RBMGAUSSIAN);
                else if (v0 == "RBMProduct") c.elements.push_back(E_RBMPRODUCT);
                else if (v0 == "hydrogenLike") c.elements.push_back(E_HYDROGENLIKE);
                else if (v0 == "hardCoreJastrow") c.elements.push_back(E_OTHER);
                else if (v0 == "mlpJastrow") c.elements.push_back(E_MLP);  // engine element
                else return err("Wave function element '" + v0 + "' does not exist!");
            } else if (key == "interactionStyle") {
                if (v0 == "noInteraction") c.coulomb = false;
                else if (v0 == "coulomb") c.coulomb = true;
                else return err("Interaction style '" + v0 + "' does not exist!");
            } else if (key == "rng") {
                if (v0 != "MersenneTwister" && v0 != "Philox")
                    return err("Random number generator '" + v0 + "' does not exist!");
                if (v.size() > 1) {
                    c.have_seed = true;
                    c.seed = std::stoll(v[1]);
                }
            } else if (key == "numWalkers") {
                c.walkers = std::stoi(v0);
            } else if (key == "driftLimit") {
                c.drift_limit = std::stod(v0);
                if (!(c.drift_limit >= 0.0)) return err("driftLimit must be >= 0");
            } else if (key == "walkerOffset") {
                c.walker_offset = std::stoi(v0);
                if (c.walker_offset < 0) return err("walkerOffset must be >= 0");
            } else if (key == "precision") {
                if (v0 == "fp64") c.precision = 0;
                else if (v0 == "mixed") c.precision = 1;
                else return err("precision must be fp64 or mixed");
            } else if (key == "refreshInterval") {
                c.refresh_interval = (v0 == "auto") ? -1 : std::stoi(v0);
            } else if (key == "mlpTensorCores") {
                if (v0 == "true") c.mlp_tc = true;
                else if (v0 == "false") c.mlp_tc = false;
                else return err("mlpTensorCores must be true or false");
            } else if (key == "compat") {
                if (v0 == "reference") c.compat = 1;
                else if (v0 == "corrected") c.compat = 0;
                else return err("compat must be reference or corrected");
            } else if (key == "walkersPerBlock") {
                c.walkers_per_block = std::stoi(v0);
            } else if (key == "walkersPerWarp") {
                if (v0 == "auto") c.walkers_per_warp = 0;
                else if (v0 == "1" || v0 == "2" || v0 == "4") c.walkers_per_warp = std::stoi(v0);
                else return err("walkersPerWarp must be auto, 1, 2 or 4");
            } else if (key == "sweepForm") {
                if (v0 == "auto") c.sweep_form = 0;
                else if (v0 == "staged") c.sweep_form = 1;
                else if (v0 == "owner") c.sweep_form = 2;
                else return err("sweepForm must be auto, staged or owner");
            } else if (key == "seed") {
                c.have_seed = true;
                c.seed = std::stoll(v0);
            } else {
                return err("Invalid key '" + key + "' is passed to configuration file!");
            }
        } catch (const std::exception &) {
            return err("bad value for '" + key + "'");
        }
    }
    c.trial_label = trial_label(c.elements);
    return "";
}

}  // namespace vmc

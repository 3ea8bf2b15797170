// b200_vmc: VMaChine's main() (src/main.cpp) with the B200 engine.
//
//   b200_vmc <input.in> engine <iterations> <seed>
//       the walker population on the GPU: B200Engine samples every iteration and
//       B200Optimization hands the optimiser's step to a System-side parameter copy as
//       `m_parameters -= m_optimization->updateParameters()` (system.cpp:114) does;
//       one JSON line per iteration
//   b200_vmc <input.in> metropolis
//       the reference's System::runSimulation, unchanged, with its Metropolis replaced
//       by B200Metropolis (System's walker moved on the GPU, on System's random numbers)
//   b200_vmc <input.in> reference
//       the reference's System::runSimulation as its own main() runs it
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <sstream>
#include <string>

#include "b200engine.h"
#include "system.h"

namespace {

std::string read_file(const char *path)
{
    std::ifstream in(path);
    std::stringstream s;
    s << in.rdbuf();
    return s.str();
}

// main.cpp: the defaults the reference's own main() sets before reading the config
void configure(System &base, const char *path)
{
    base.setNumberOfParticles(2);
    base.setNumberOfDimensions(2);
    base.setEquilibrationFraction(0.001);
    char prog[] = "b200_vmc";
    char *argv[] = {prog, const_cast<char *>(path), nullptr};
    base.initializeFromConfig(2, argv);
}

int run_engine(const std::string &text, int iterations, uint64_t seed)
{
    B200Engine engine(text);
    engine.initializeWalkers(seed);
    System system;  // the System whose parameters the stand-in optimiser keeps in step
    B200Optimization optimization(&system, &engine);
    Eigen::MatrixXd parameters = engine.parameters();
    for (int it = 0; it < iterations; ++it) {
        const vmc_averages a = optimization.iterate(it);
        parameters -= optimization.updateParameters();
        const double gap = (parameters - engine.parameters()).cwiseAbs().maxCoeff();
        std::printf("{\"iteration\": %d, \"energy\": %.17g, \"std_error\": %.17g, \"acceptance\": %.17g, "
                    "\"kinetic\": %.17g, \"parameter_gap\": %.3g}\n",
                    it, a.energy, a.std_error, a.acceptance, a.kinetic, gap);
    }
    return 0;
}

}  // namespace

int main(int argc, char **argv)
{
    if (argc < 3) {
        std::fprintf(stderr, "usage: %s <input.in> engine <iterations> <seed> | metropolis | reference\n", argv[0]);
        return 2;
    }
    const std::string mode = argv[2];
    try {
        if (mode == "engine") {
            const int iterations = argc > 3 ? std::atoi(argv[3]) : 3;
            const uint64_t seed = argc > 4 ? std::strtoull(argv[4], nullptr, 10) : 1;
            return run_engine(read_file(argv[1]), iterations, seed);
        }
        System base;
        configure(base, argv[1]);
        if (mode == "metropolis") base.setMetropolis(new B200Metropolis(&base, read_file(argv[1])));
        else if (mode != "reference") return 2;
        base.runSimulation();
    } catch (const B200Error &e) {
        std::fprintf(stderr, "b200 engine error %d: %s\n", e.code, e.message.c_str());
        return 1;
    }
    return 0;
}

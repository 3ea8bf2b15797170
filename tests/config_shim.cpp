// Test shim (test infrastructure only): the engine's input.in parser
// (vmachine_b200/csrc/vmc_config.cpp) built for the host, so CPU tests can read what
// it makes of a configuration without a GPU.
#include "vmc_config.hpp"

#include <cstring>
#include <string>

extern "C" long cfg_trial_label(const char *text, char *buf, long cap)
{
    vmc::Config c;
    if (!vmc::parse_config(text, c).empty()) return -1;
    if ((long)c.trial_label.size() + 1 > cap) return -2;
    std::memcpy(buf, c.trial_label.c_str(), c.trial_label.size() + 1);
    return (long)c.trial_label.size();
}

// The parsed settings in the order of the reference harness's vmref_settings.
extern "C" int cfg_settings(const char *text, double *out)
{
    vmc::Config c;
    if (!vmc::parse_config(text, c).empty()) return -1;
    const double v[] = {double(c.N), double(c.dim), c.omega, c.sigma, double(c.Z), double(c.hidden), c.eta,
                        double(c.iterations), c.eq_fraction, double(c.num_steps), c.step_length,
                        double(c.sorting), c.max_radius, double(c.n_bins), c.tolerance,
                        double(c.n_energies), double(c.range_adaptive), double(c.add_steps),
                        double(c.add_steps_last), double(c.checkpoint_freq), double(c.check_convergence),
                        double(c.adaptive_steps), double(c.ob_density), double(c.ob_density2),
                        double(c.tb_density)};
    const int n = int(sizeof(v) / sizeof(v[0]));
    for (int i = 0; i < n; i++) out[i] = v[i];
    return n;
}

// Per-element parameter counts of the parsed configuration, in element order.
// Returns the number of elements, or -1 if the text does not parse.
extern "C" int cfg_parameter_counts(const char *text, int *out, int cap)
{
    vmc::Config c;
    if (!vmc::parse_config(text, c).empty()) return -1;
    const int n = (int)c.elements.size();
    for (int i = 0; i < n && i < cap; i++) out[i] = vmc::element_parameters(c, c.elements[i]);
    return n;
}

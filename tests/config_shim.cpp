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

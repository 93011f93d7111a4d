// codegen.h -- CUDA source generation for one circuit + solve configuration.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "lutmap.h"

namespace nsat {

enum class Mode { SAT = 1, QSAT = 2, TABLE = 3 };

struct KernelConfig {
    Mode mode = Mode::SAT;
    uint32_t nin = 0;          // circuit inputs, padding included
    uint32_t nb = 0;           // enumeration bits (== nin)
    std::vector<int> in_of_bit;  // enumeration bit -> circuit input
    uint32_t it = 0, wb = 0, cb = 0;  // log2 iterations/warp, warps/CTA, CTAs/launch
    uint32_t minb = 0;         // __launch_bounds__ minimum CTAs per SM (0 = none)
    uint32_t sync_every = 0;   // SAT/QSAT: CTA barrier after every this many LUTs (0 = none)
    uint32_t c = 0;            // 10 + it + wb + cb
    // QSAT
    uint32_t m = 0;            // unit level (inner bits below the first block)
    bool q0all = false;
    uint64_t allbits = 0;      // enumeration bit j quantifier is All
    bool data = false;         // items from a buffer (reduction tests)
    // TABLE
    uint32_t fmt = 0;          // 0 u32, 1 u64, 2 u64 + distance
    uint32_t nout = 1;

    uint32_t threads() const { return 32u << wb; }
    std::string key() const;   // every field the generated source depends on (with the LUT net)
};

// Full NVRTC source: prelude, generated input/eval functions, template.
std::string generate_source(const KernelConfig& kc, const LutNet& net);

// The template text (device_template.cuh), embedded at build time.
extern const char* const kDeviceTemplate;

}  // namespace nsat

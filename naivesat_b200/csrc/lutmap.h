// lutmap.h -- cover a two-input gate circuit with 3-input LUTs (lop3.b32).
//
// A 3-input LUT is exactly what one lop3.b32 instruction computes, so the
// number of LUTs is the number of logic instructions per 32-lane word.  The
// mapper enumerates cuts with their truth tables, reduces each to the support
// of its function, picks 3-leaf cuts by area flow (Cong & Ding style priority
// cuts), then does exact-area recovery passes.  Negations never cost an
// instruction: they live in the truth tables.  A node whose function is
// constant becomes a LUT with a constant table that reads input 0.
#pragma once
#include <cstdint>
#include <vector>

#include "circuit.h"

namespace nsat {

struct Lut {
    uint32_t wire;       // circuit wire this LUT computes
    uint8_t nin;         // 1..3 leaves (a constant LUT has 1, input 0, ignored)
    uint32_t in[3];      // leaf wires (operands a, b, c of lop3)
    uint8_t tt;          // lop3 immediate: f(a,b,c) = bit (a<<2 | b<<1 | c)
};

struct LutNet {
    std::vector<Lut> luts;               // topological order
    std::vector<uint32_t> used_inputs;   // circuit inputs read by some LUT/output
    std::vector<Output> outs;            // requested outputs: wire (+ negation)
    uint32_t live_gates = 0;             // gates in the cone of the outputs
};

// Maps the cone of outputs `which` (indices into c.outputs).  With
// one_per_gate, every live gate becomes its own 2-leaf LUT (no fusion).
// recovery_passes: exact-area recovery passes over the cover (the second
// rarely saves more than a LUT).
// cut_leaves (3..6) bounds the cuts enumerated before support reduction:
// wider finds smaller covers and costs more time.  On the 3000-gate random
// DAGs of the benchmarks, three leaves take about 3 ms and six about 27 ms
// for 4-6 % fewer LUTs.
LutNet map_luts(const Circuit& c, const std::vector<uint32_t>& which, bool one_per_gate, int cut_leaves,
                int recovery_passes = 2);

// Gates in the cone of outputs `which`.
uint32_t live_gate_count(const Circuit& c, const std::vector<uint32_t>& which);

// The cover for a search of 2^log2_space assignments evaluated at about
// `lut_words_per_s`.  For a solve that has the device to itself: when even
// one LUT per live gate would search in under a quarter of the time that cut
// mapping takes (small index spaces: the 2^24 search of a 500-gate circuit is
// about 8 us of lop3 work against about 0.3 ms of mapping), the cover is one
// LUT per gate, a linear pass.  With `shared_device` (jobs of a server, whose
// device time every other job waits for) that shortcut is not taken.
// Otherwise it maps with three leaves, estimates the search's time from that
// cover, and maps again with wider cuts only when the expected saving beats
// the extra mapping time (the width minimising mapping plus search).
LutNet map_luts_for(const Circuit& c, const std::vector<uint32_t>& which, bool one_per_gate, double log2_space,
                    double lut_words_per_s, bool shared_device = false);
constexpr double kCompiledLutWordsPerS = 1.85e13;   // compiled kernels: the lop3 issue rate of a B200
constexpr double kServedLutWordsPerS = 2.0e12;      // the serving interpreter

// Reference evaluation of a LutNet on 32-lane words (used by host self-checks).
void eval_lutnet32(const LutNet& net, uint32_t nwires, const uint32_t* inputs, uint32_t* outs);

}  // namespace nsat

// lutmap.h -- cover a two-input gate circuit with 3-input LUTs (lop3.b32).
//
// A 3-input LUT is exactly what one lop3.b32 instruction computes, so the
// number of LUTs is the number of logic instructions per 32-lane word.  The
// mapper enumerates cuts of at most 3 leaves per node, picks cuts by area flow
// (Cong & Ding style priority cuts), then does exact-area recovery passes.
// Negations never cost an instruction: they live in the truth tables.
#pragma once
#include <cstdint>
#include <vector>

#include "circuit.h"

namespace nsat {

struct Lut {
    uint32_t wire;       // circuit wire this LUT computes
    uint8_t nin;         // 1..3 leaves
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
LutNet map_luts(const Circuit& c, const std::vector<uint32_t>& which, bool one_per_gate);

// Reference evaluation of a LutNet on 32-lane words (used by host self-checks).
void eval_lutnet32(const LutNet& net, uint32_t nwires, const uint32_t* inputs, uint32_t* outs);

}  // namespace nsat

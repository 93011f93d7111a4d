// circuit.h -- host-side Gate circuit IR, validation and gatesim text I/O.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace nsat {

enum GateFunc : uint8_t { AND = 0, NOR = 1, NIMPL = 2, XOR = 3 };

struct Gate {
    uint8_t func;
    uint32_t i0, i1;
};

struct Output {
    uint32_t wire;
    bool neg;
};

// Two-input gate circuit in gatesim's shape (Circuit::new(n, gates, outputs)):
// wires 0..n-1 are inputs, wire n+k is gates[k].
struct Circuit {
    uint32_t n = 0;
    std::vector<Gate> gates;
    std::vector<Output> outputs;

    uint32_t wires() const { return n + (uint32_t)gates.size(); }
    // Returns an empty string if valid, else the reason.
    std::string validate() const;
    // 64-bit FNV-1a content hash (used as the JIT cache key component).
    uint64_t hash() const;
};

// Truth table of a gate function over (i0, i1) with i0 = bit 1, i1 = bit 0
// of the row index: bit r of the result is f(r>>1 & 1, r & 1).
uint8_t gate_tt2(uint8_t func);
// Applies gate func to whole words.
inline uint32_t gate_eval32(uint8_t f, uint32_t a, uint32_t b) {
    switch (f) {
    case AND: return a & b;
    case NOR: return ~(a | b);
    case NIMPL: return a & ~b;
    default: return a ^ b;
    }
}

// gatesim text format, reconstructed from gatesim's documentation (the crate
// is not vendored, so no reference file pins this grammar):
//   [quantifiers] '{' tokens '}' '(' n ')'
// tokens are input indices or gates `and(a,b)`, `nor(a,b)`, `nimpl(a,b)`,
// `xor(a,b)`, each optionally followed by output markers `:k` or `:kn`
// (n = negated).  Gates are numbered n, n+1, ... in order of appearance.
// The optional quantifier prefix lists one of a/e (A/E) per input.
struct Parsed {
    Circuit circuit;
    std::vector<uint8_t> quants;  // empty if none; 1 = All
};
bool parse_gatesim(const std::string& text, Parsed* out, std::string* err);
std::string format_gatesim(const Circuit& c, const std::vector<uint8_t>* quants);

}  // namespace nsat

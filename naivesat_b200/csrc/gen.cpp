// gen.cpp -- seeded synthetic circuits of the benchmark configurations
// (random DAGs, LFSR+mixer next-state circuits), bit-identical to the
// Python generators in naivesat_b200/workloads.py: splitmix64 draws,
// rejection-sampled ranges, fan-in negations folded into AND/NOR/NIMPL/XOR.
#include <cstdint>
#include <cstring>
#include <set>
#include <vector>

#include "circuit.h"
#include "nsat.h"

using namespace nsat;

namespace {

struct SplitMix64 {
    uint64_t s;
    explicit SplitMix64(uint64_t seed) : s(seed) {}
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ull;
        uint64_t z = s;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    }
    uint64_t below(uint64_t k) {
        if (k <= 1) return 0;
        // lim = 2^64 - (2^64 mod k), computed without 128-bit arithmetic
        const uint64_t rem = (uint64_t)(((unsigned __int128)1 << 64) % k);
        const unsigned __int128 lim = ((unsigned __int128)1 << 64) - rem;
        for (;;) {
            uint64_t v = next();
            if ((unsigned __int128)v < lim) return v % k;
        }
    }
};

struct Raw {
    uint8_t f;
    uint32_t a, b;
    uint8_t na, nb;
};

struct RawBuilder {
    uint32_t n;
    std::vector<Raw> raw;
    std::vector<std::pair<uint32_t, uint8_t>> outs;
    explicit RawBuilder(uint32_t nin) : n(nin) {}
    uint32_t gate(uint8_t f, uint32_t a, uint32_t b, uint8_t na = 0, uint8_t nb = 0) {
        raw.push_back(Raw{f, a, b, na, nb});
        return n + (uint32_t)raw.size() - 1;
    }
};

uint32_t g2(uint8_t f, uint32_t x, uint32_t y) { return gate_eval32(f, x ? 1u : 0u, y ? 1u : 0u) & 1u; }

// (func, negate i0, negate i1) -> (func, swap, complement), the first match
// in the order func, AND, NOR, NIMPL, XOR x swap 0,1 x complement 0,1.
void canon(uint8_t f, uint8_t ea, uint8_t eb, uint8_t* g, uint8_t* swap, uint8_t* oneg) {
    uint32_t tt[4];
    for (uint32_t x = 0; x < 2; x++)
        for (uint32_t y = 0; y < 2; y++) tt[2 * x + y] = g2(f, x ^ ea, y ^ eb);
    const uint8_t order[5] = {f, AND, NOR, NIMPL, XOR};
    for (uint8_t gi : order)
        for (uint8_t sw = 0; sw < 2; sw++)
            for (uint8_t on = 0; on < 2; on++) {
                bool ok = true;
                for (uint32_t x = 0; x < 2 && ok; x++)
                    for (uint32_t y = 0; y < 2 && ok; y++)
                        ok = ((sw ? g2(gi, y, x) : g2(gi, x, y)) ^ on) == tt[2 * x + y];
                if (ok) { *g = gi; *swap = sw; *oneg = on; return; }
            }
}

Circuit fold(const RawBuilder& rb) {
    Circuit c;
    c.n = rb.n;
    std::vector<uint8_t> inv(rb.n + rb.raw.size(), 0);
    for (size_t k = 0; k < rb.raw.size(); k++) {
        const Raw& r = rb.raw[k];
        uint8_t g = AND, sw = 0, on = 0;
        canon(r.f, r.na ^ inv[r.a], r.nb ^ inv[r.b], &g, &sw, &on);
        c.gates.push_back(sw ? Gate{g, r.b, r.a} : Gate{g, r.a, r.b});
        inv[rb.n + k] = on;
    }
    for (auto& o : rb.outs) c.outputs.push_back(Output{o.first, (o.second ^ inv[o.first]) != 0});
    return c;
}

void random_dag_raw(SplitMix64& rng, RawBuilder& rb, uint32_t gates, uint32_t window) {
    const uint32_t n = rb.n;
    for (uint32_t k = 0; k < gates; k++) {
        const uint32_t node = n + k;
        const uint32_t lo = node > window ? node - window : 0;
        const uint8_t f = (uint8_t)rng.below(4);
        const uint32_t a = lo + (uint32_t)rng.below(node - lo);
        const uint8_t na = rng.below(4) == 0;
        const uint32_t b = lo + (uint32_t)rng.below(node - lo);
        const uint8_t nb = rng.below(4) == 0;
        rb.gate(f, a, b, na, nb);
    }
}

// Last gate whose value is not constant on 4096 seeded samples.
uint32_t last_live_gate(const Circuit& c) {
    SplitMix64 rng(0x5A3B1E);
    const int K = 64;
    std::vector<uint64_t> w((size_t)(c.n + c.gates.size()) * K);
    for (uint32_t i = 0; i < c.n; i++)
        for (int k = 0; k < K; k++) w[(size_t)i * K + k] = rng.next();
    for (size_t g = 0; g < c.gates.size(); g++) {
        const Gate& G = c.gates[g];
        uint64_t* d = &w[(c.n + g) * K];
        const uint64_t* x = &w[(size_t)G.i0 * K];
        const uint64_t* y = &w[(size_t)G.i1 * K];
        for (int k = 0; k < K; k++) {
            switch (G.func) {
            case AND: d[k] = x[k] & y[k]; break;
            case NOR: d[k] = ~(x[k] | y[k]); break;
            case NIMPL: d[k] = x[k] & ~y[k]; break;
            default: d[k] = x[k] ^ y[k]; break;
            }
        }
    }
    for (size_t g = c.gates.size(); g-- > 0;) {
        const uint64_t* d = &w[(c.n + g) * K];
        bool zero = true, ones = true;
        for (int k = 0; k < K; k++) { zero &= d[k] == 0; ones &= d[k] == ~0ull; }
        if (!zero && !ones) return (uint32_t)g;
    }
    return (uint32_t)c.gates.size() - 1;
}

int emit(const Circuit& c, uint32_t* gates, uint32_t gate_cap, uint32_t* outputs, uint32_t out_cap,
         uint32_t* gate_num, uint32_t* out_num) {
    *gate_num = (uint32_t)c.gates.size();
    *out_num = (uint32_t)c.outputs.size();
    if (c.gates.size() > gate_cap || c.outputs.size() > out_cap) return NSAT_EINVAL;
    for (size_t k = 0; k < c.gates.size(); k++) {
        gates[3 * k] = c.gates[k].func; gates[3 * k + 1] = c.gates[k].i0; gates[3 * k + 2] = c.gates[k].i1;
    }
    for (size_t j = 0; j < c.outputs.size(); j++) { outputs[2 * j] = c.outputs[j].wire; outputs[2 * j + 1] = c.outputs[j].neg; }
    return NSAT_OK;
}

}  // namespace

extern "C" int nsat_gen_random_dag(uint64_t seed, uint32_t n, uint32_t gates, uint32_t window, int live_output,
                                   uint32_t* out_gates, uint32_t gate_cap, uint32_t* out_outputs,
                                   uint32_t out_cap, uint32_t* gate_num, uint32_t* out_num) {
    if (n == 0 || gates == 0 || !out_gates || !out_outputs || !gate_num || !out_num) return NSAT_EINVAL;
    SplitMix64 rng(seed);
    RawBuilder rb(n);
    random_dag_raw(rng, rb, gates, window);
    uint32_t out = n + gates - 1;
    if (live_output) {
        rb.outs.push_back({out, 0});
        Circuit probe = fold(rb);
        rb.outs.clear();
        out = n + last_live_gate(probe);
    }
    rb.outs.push_back({out, 0});
    return emit(fold(rb), out_gates, gate_cap, out_outputs, out_cap, gate_num, out_num);
}

extern "C" int nsat_gen_lfsr_stop(uint64_t seed, uint32_t n, uint32_t mixer_gates, uint32_t* out_gates,
                                  uint32_t gate_cap, uint32_t* out_outputs, uint32_t out_cap, uint32_t* gate_num,
                                  uint32_t* out_num, uint64_t* pattern_out) {
    if (n < 4 || n > 63 || mixer_gates < n || !out_gates || !out_outputs) return NSAT_EINVAL;
    SplitMix64 rng(seed);
    std::set<uint32_t> taps{n - 1};
    while (taps.size() < 4) taps.insert((uint32_t)rng.below(n - 1));
    std::vector<uint32_t> tv(taps.begin(), taps.end());
    const uint64_t pattern = rng.next() & ((1ull << n) - 1);
    RawBuilder rb(n);
    random_dag_raw(rng, rb, mixer_gates, 64);
    const uint32_t mix_first = n + (mixer_gates - n);
    uint32_t fb = rb.gate(XOR, tv[0], tv[1]);
    for (size_t t = 2; t < tv.size(); t++) fb = rb.gate(XOR, fb, tv[t]);
    std::vector<uint32_t> nxt;
    for (uint32_t i = 0; i < n; i++) nxt.push_back(rb.gate(XOR, i == 0 ? fb : i - 1, mix_first + i));
    uint32_t acc = rb.gate(AND, 0, 1, (pattern & 1) ? 0 : 1, ((pattern >> 1) & 1) ? 0 : 1);
    for (uint32_t i = 2; i < n; i++) acc = rb.gate(AND, acc, i, 0, ((pattern >> i) & 1) ? 0 : 1);
    for (uint32_t w : nxt) rb.outs.push_back({w, 0});
    rb.outs.push_back({acc, 0});
    if (pattern_out) *pattern_out = pattern;
    return emit(fold(rb), out_gates, gate_cap, out_outputs, out_cap, gate_num, out_num);
}

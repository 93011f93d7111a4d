// lutmap.cpp -- priority-cut 3-LUT mapping with area flow and exact-area recovery.
#include "lutmap.h"

#include <algorithm>
#include <unordered_map>

namespace nsat {

namespace {

constexpr int K = 3;          // LUT inputs (lop3)
constexpr int P = 10;         // cuts kept per node

struct Cut {
    uint8_t n = 0;
    uint32_t l[K];
    float af = 0;
    bool operator==(const Cut& o) const {
        if (n != o.n) return false;
        for (int i = 0; i < n; i++) if (l[i] != o.l[i]) return false;
        return true;
    }
};

// merge two sorted leaf sets; false if more than K leaves
bool merge(const Cut& a, const Cut& b, Cut* out) {
    int i = 0, j = 0, k = 0;
    while (i < a.n || j < b.n) {
        uint32_t v;
        if (j >= b.n || (i < a.n && a.l[i] < b.l[j])) v = a.l[i++];
        else if (i >= a.n || b.l[j] < a.l[i]) v = b.l[j++];
        else { v = a.l[i]; i++; j++; }
        if (k == K) return false;
        out->l[k++] = v;
    }
    out->n = (uint8_t)k;
    return true;
}

struct Mapper {
    const Circuit& c;
    uint32_t n, W;
    std::vector<uint8_t> live;
    std::vector<uint32_t> fanout;
    std::vector<std::vector<Cut>> cuts;   // per wire (gates only non-empty)
    std::vector<Cut> best;
    std::vector<float> af;
    std::vector<int32_t> refs;

    explicit Mapper(const Circuit& cc) : c(cc), n(cc.n), W(cc.wires()) {}

    bool is_gate(uint32_t w) const { return w >= n; }
    const Gate& gate(uint32_t w) const { return c.gates[w - n]; }

    int ref_cut(const Cut& cut) {
        int area = 1;
        for (int i = 0; i < cut.n; i++) {
            uint32_t l = cut.l[i];
            if (is_gate(l) && refs[l]++ == 0) area += ref_cut(best[l]);
        }
        return area;
    }
    int deref_cut(const Cut& cut) {
        int area = 1;
        for (int i = 0; i < cut.n; i++) {
            uint32_t l = cut.l[i];
            if (is_gate(l) && --refs[l] == 0) area += deref_cut(best[l]);
        }
        return area;
    }

    void enumerate() {
        cuts.assign(W, {});
        best.assign(W, Cut());
        af.assign(W, 0.f);
        for (uint32_t w = n; w < W; w++) {
            if (!live[w]) continue;
            const Gate& g = gate(w);
            auto fanin_cuts = [&](uint32_t x) {
                std::vector<Cut> v;
                Cut triv; triv.n = 1; triv.l[0] = x; triv.af = is_gate(x) ? af[x] : 0.f;
                v.push_back(triv);
                if (is_gate(x)) for (const Cut& ct : cuts[x]) if (!(ct.n == 1 && ct.l[0] == x)) v.push_back(ct);
                return v;
            };
            std::vector<Cut> ca = fanin_cuts(g.i0), cb = fanin_cuts(g.i1);
            std::vector<Cut> cand;
            for (const Cut& x : ca)
                for (const Cut& y : cb) {
                    Cut m;
                    if (!merge(x, y, &m)) continue;
                    if (std::find(cand.begin(), cand.end(), m) != cand.end()) continue;
                    float a = 1.f;
                    for (int i = 0; i < m.n; i++) {
                        uint32_t l = m.l[i];
                        if (is_gate(l)) a += af[l] / (float)std::max<uint32_t>(1, fanout[l]);
                    }
                    m.af = a;
                    cand.push_back(m);
                }
            std::stable_sort(cand.begin(), cand.end(), [](const Cut& x, const Cut& y) {
                if (x.af != y.af) return x.af < y.af;
                return x.n < y.n;
            });
            if ((int)cand.size() > P) cand.resize(P);
            best[w] = cand[0];
            af[w] = cand[0].af;
            cuts[w] = cand;
        }
    }
};

uint8_t cone_tt(const Circuit& c, uint32_t root, const uint32_t* leaves, int nl,
                std::unordered_map<uint32_t, uint8_t>& memo) {
    static const uint8_t pat[3] = {0xF0, 0xCC, 0xAA};
    memo.clear();
    for (int i = 0; i < nl; i++) memo[leaves[i]] = pat[i];
    // iterative post-order over the cone
    std::vector<uint32_t> stack{root};
    while (!stack.empty()) {
        uint32_t w = stack.back();
        if (memo.count(w)) { stack.pop_back(); continue; }
        const Gate& g = c.gates[w - c.n];
        bool ready = true;
        if (!memo.count(g.i0)) { stack.push_back(g.i0); ready = false; }
        if (!memo.count(g.i1)) { stack.push_back(g.i1); ready = false; }
        if (!ready) continue;
        stack.pop_back();
        memo[w] = (uint8_t)gate_eval32(g.func, memo[g.i0], memo[g.i1]);
    }
    return memo[root];
}

}  // namespace

LutNet map_luts(const Circuit& c, const std::vector<uint32_t>& which, bool one_per_gate) {
    LutNet net;
    Mapper m(c);
    const uint32_t n = c.n, W = c.wires();
    m.live.assign(W, 0);
    for (uint32_t j : which) m.live[c.outputs[j].wire] = 1;
    for (int64_t w = (int64_t)W - 1; w >= (int64_t)n; w--)
        if (m.live[w]) { m.live[m.gate((uint32_t)w).i0] = 1; m.live[m.gate((uint32_t)w).i1] = 1; }
    m.fanout.assign(W, 0);
    for (uint32_t w = n; w < W; w++)
        if (m.live[w]) { m.fanout[m.gate(w).i0]++; m.fanout[m.gate(w).i1]++; }
    for (uint32_t j : which) m.fanout[c.outputs[j].wire]++;
    for (uint32_t w = n; w < W; w++) net.live_gates += m.live[w];

    if (one_per_gate) {
        for (uint32_t w = n; w < W; w++) {
            if (!m.live[w]) continue;
            Cut ct;
            const Gate& g = m.gate(w);
            ct.n = 0;
            ct.l[ct.n++] = g.i0;
            if (g.i1 != g.i0) ct.l[ct.n++] = g.i1;
            m.best.resize(W);
            m.best[w] = ct;
        }
        m.best.resize(W);
        m.refs.assign(W, 0);
    } else {
        m.enumerate();
        // initial cover from area-flow choices
        m.refs.assign(W, 0);
        for (uint32_t j : which) {
            uint32_t w = c.outputs[j].wire;
            if (m.is_gate(w) && m.refs[w]++ == 0) m.ref_cut(m.best[w]);
        }
        // exact-area recovery (two passes)
        for (int pass = 0; pass < 2; pass++) {
            for (uint32_t w = n; w < W; w++) {
                if (!m.live[w] || m.refs[w] <= 0) continue;
                m.deref_cut(m.best[w]);
                int best_area = 1 << 30;
                size_t best_i = 0;
                for (size_t i = 0; i < m.cuts[w].size(); i++) {
                    const Cut& ct = m.cuts[w][i];
                    int a = m.ref_cut(ct);
                    m.deref_cut(ct);
                    if (a < best_area) { best_area = a; best_i = i; }
                }
                m.best[w] = m.cuts[w][best_i];
                m.ref_cut(m.best[w]);
            }
        }
    }

    // collect the cover: roots are the outputs; walk selected cuts
    std::vector<uint8_t> need(W, 0);
    for (uint32_t j : which) need[c.outputs[j].wire] = 1;
    for (int64_t w = (int64_t)W - 1; w >= (int64_t)n; w--) {
        if (!need[w]) continue;
        const Cut& ct = m.best[w];
        for (int i = 0; i < ct.n; i++) need[ct.l[i]] = 1;
    }
    std::unordered_map<uint32_t, uint8_t> memo;
    for (uint32_t w = n; w < W; w++) {
        if (!need[w]) continue;
        const Cut& ct = m.best[w];
        Lut L;
        L.wire = w;
        L.nin = ct.n;
        for (int i = 0; i < K; i++) L.in[i] = i < ct.n ? ct.l[i] : ct.l[0];
        L.tt = cone_tt(c, w, ct.l, ct.n, memo);
        net.luts.push_back(L);
    }
    for (uint32_t i = 0; i < n; i++) if (need[i]) net.used_inputs.push_back(i);
    for (uint32_t j : which) net.outs.push_back(c.outputs[j]);
    return net;
}

void eval_lutnet32(const LutNet& net, uint32_t nwires, const uint32_t* inputs, uint32_t* outs) {
    std::vector<uint32_t> v(nwires, 0);
    for (uint32_t i : net.used_inputs) v[i] = inputs[i];
    for (const Lut& L : net.luts) {
        uint32_t a = v[L.in[0]], b = v[L.in[1]], cc = v[L.in[2]];
        uint32_t r = 0;
        for (int row = 0; row < 8; row++) {
            if (!((L.tt >> row) & 1)) continue;
            uint32_t ma = (row & 4) ? a : ~a, mb = (row & 2) ? b : ~b, mc = (row & 1) ? cc : ~cc;
            r |= ma & mb & mc;
        }
        v[L.wire] = r;
    }
    for (size_t j = 0; j < net.outs.size(); j++)
        outs[j] = v[net.outs[j].wire] ^ (net.outs[j].neg ? ~0u : 0u);
}

}  // namespace nsat

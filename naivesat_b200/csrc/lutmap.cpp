// lutmap.cpp -- priority-cut 3-LUT mapping with area flow and exact-area recovery.
#include "lutmap.h"

#include <algorithm>

namespace nsat {

namespace {

constexpr int K = 3;          // LUT inputs (lop3)
constexpr int P = 10;         // cuts kept per node

struct Cut {
    uint8_t n = 0;
    uint32_t l[K];
    uint32_t sig = 0;   // OR of 1 << (leaf % 32): more than K bits set means more than K leaves
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
    out->sig = a.sig | b.sig;
    return true;
}

struct Mapper {
    const Circuit& c;
    uint32_t n, W;
    std::vector<uint8_t> live;
    std::vector<uint32_t> fanout;
    std::vector<Cut> cuts;      // gate w's kept cuts: cuts[(w - n) * P .. + ncut[w - n])
    std::vector<uint8_t> ncut;
    std::vector<Cut> best;
    std::vector<float> af;
    std::vector<int32_t> refs;
    std::vector<uint32_t> stk;  // work list of ref_cut / deref_cut
    std::vector<uint32_t> log;  // reference increments made by ref_cut_bounded

    explicit Mapper(const Circuit& cc) : c(cc), n(cc.n), W(cc.wires()) {}

    bool is_gate(uint32_t w) const { return w >= n; }
    const Gate& gate(uint32_t w) const { return c.gates[w - n]; }
    const Cut* cuts_of(uint32_t w) const { return &cuts[(size_t)(w - n) * P]; }

    // References the cut's leaves; every gate whose count leaves 0 joins the
    // cover with its best cut.  Returns the LUTs added (the cut's own included).
    int ref_cut(const Cut& cut) {
        int area = 1;
        stk.clear();
        for (int i = 0; i < cut.n; i++)
            if (is_gate(cut.l[i]) && refs[cut.l[i]]++ == 0) stk.push_back(cut.l[i]);
        while (!stk.empty()) {
            const uint32_t x = stk.back();
            stk.pop_back();
            area++;
            const Cut& b = best[x];
            for (int i = 0; i < b.n; i++)
                if (is_gate(b.l[i]) && refs[b.l[i]]++ == 0) stk.push_back(b.l[i]);
        }
        return area;
    }
    // ref_cut for comparing candidates: stops counting once the area
    // reaches `limit` (the candidate cannot win then; a smaller count is
    // exact) and logs every increment for undo_log().
    int ref_cut_bounded(const Cut& cut, int limit) {
        int area = 1;
        stk.clear();
        log.clear();
        for (int i = 0; i < cut.n; i++)
            if (is_gate(cut.l[i])) {
                log.push_back(cut.l[i]);
                if (refs[cut.l[i]]++ == 0) stk.push_back(cut.l[i]);
            }
        while (!stk.empty() && area < limit) {
            const uint32_t x = stk.back();
            stk.pop_back();
            area++;
            const Cut& b = best[x];
            for (int i = 0; i < b.n; i++)
                if (is_gate(b.l[i])) {
                    log.push_back(b.l[i]);
                    if (refs[b.l[i]]++ == 0) stk.push_back(b.l[i]);
                }
        }
        return area;
    }
    void undo_log() {
        for (uint32_t x : log) refs[x]--;
    }
    // The inverse of ref_cut: returns the LUTs removed.
    int deref_cut(const Cut& cut) {
        int area = 1;
        stk.clear();
        for (int i = 0; i < cut.n; i++)
            if (is_gate(cut.l[i]) && --refs[cut.l[i]] == 0) stk.push_back(cut.l[i]);
        while (!stk.empty()) {
            const uint32_t x = stk.back();
            stk.pop_back();
            area++;
            const Cut& b = best[x];
            for (int i = 0; i < b.n; i++)
                if (is_gate(b.l[i]) && --refs[b.l[i]] == 0) stk.push_back(b.l[i]);
        }
        return area;
    }

    // A fanin's cuts: its trivial cut first, then its kept cuts.
    int fanin_cuts(uint32_t x, Cut* v) const {
        int k = 0;
        Cut& triv = v[k++];
        triv.n = 1;
        triv.l[0] = x;
        triv.sig = 1u << (x & 31u);
        triv.af = is_gate(x) ? af[x] : 0.f;
        if (is_gate(x)) {
            const Cut* cx = cuts_of(x);
            for (int i = 0; i < ncut[x - n]; i++)
                if (!(cx[i].n == 1 && cx[i].l[0] == x)) v[k++] = cx[i];
        }
        return k;
    }

    void enumerate() {
        cuts.assign((size_t)(W - n) * P, Cut());
        ncut.assign(W - n, 0);
        best.assign(W, Cut());
        af.assign(W, 0.f);
        Cut ca[P + 1], cb[P + 1], cand[(P + 1) * (P + 1)];
        for (uint32_t w = n; w < W; w++) {
            if (!live[w]) continue;
            const Gate& g = gate(w);
            const int na = fanin_cuts(g.i0, ca), nb = fanin_cuts(g.i1, cb);
            int nc = 0;
            for (int ia = 0; ia < na; ia++)
                for (int ib = 0; ib < nb; ib++) {
                    Cut m;
                    if (__builtin_popcount(ca[ia].sig | cb[ib].sig) > K) continue;
                    if (!merge(ca[ia], cb[ib], &m)) continue;
                    bool dup = false;
                    for (int j = 0; j < nc && !dup; j++) dup = cand[j] == m;
                    if (dup) continue;
                    float a = 1.f;
                    for (int i = 0; i < m.n; i++) {
                        uint32_t l = m.l[i];
                        if (is_gate(l)) a += af[l] / (float)std::max<uint32_t>(1, fanout[l]);
                    }
                    m.af = a;
                    cand[nc++] = m;
                }
            // the P best by (area flow, leaves), ties in generation order
            Cut* keep = &cuts[(size_t)(w - n) * P];
            int nk = 0;
            for (int j = 0; j < nc; j++) {
                const Cut& x = cand[j];
                int pos = nk;
                while (pos > 0 && (x.af < keep[pos - 1].af || (x.af == keep[pos - 1].af && x.n < keep[pos - 1].n)))
                    pos--;
                if (pos >= P) continue;
                for (int k = std::min(nk, P - 1); k > pos; k--) keep[k] = keep[k - 1];
                keep[pos] = x;
                if (nk < P) nk++;
            }
            ncut[w - n] = (uint8_t)nk;
            best[w] = keep[0];
            af[w] = keep[0].af;
        }
    }
};

// Truth table of the cone from `leaves` up to `root` as a lop3 immediate.
struct ConeEval {
    std::vector<uint32_t> stamp;
    std::vector<uint8_t> val;
    std::vector<uint32_t> stack;
    uint32_t cur = 0;

    explicit ConeEval(uint32_t W) : stamp(W, 0), val(W, 0) {}

    uint8_t tt(const Circuit& c, uint32_t root, const uint32_t* leaves, int nl) {
        static const uint8_t pat[3] = {0xF0, 0xCC, 0xAA};
        cur++;
        for (int i = 0; i < nl; i++) { stamp[leaves[i]] = cur; val[leaves[i]] = pat[i]; }
        // iterative post-order over the cone
        stack.assign(1, root);
        while (!stack.empty()) {
            const uint32_t w = stack.back();
            if (stamp[w] == cur) { stack.pop_back(); continue; }
            const Gate& g = c.gates[w - c.n];
            bool ready = true;
            if (stamp[g.i0] != cur) { stack.push_back(g.i0); ready = false; }
            if (stamp[g.i1] != cur) { stack.push_back(g.i1); ready = false; }
            if (!ready) continue;
            stack.pop_back();
            stamp[w] = cur;
            val[w] = (uint8_t)gate_eval32(g.func, val[g.i0], val[g.i1]);
        }
        return val[root];
    }
};

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
                const Cut* cw = m.cuts_of(w);
                for (size_t i = 0; i < m.ncut[w - n]; i++) {
                    const Cut& ct = cw[i];
                    int a = m.ref_cut_bounded(ct, best_area);
                    m.undo_log();
                    if (a < best_area) { best_area = a; best_i = i; }
                }
                m.best[w] = cw[best_i];
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
    ConeEval cone(W);
    for (uint32_t w = n; w < W; w++) {
        if (!need[w]) continue;
        const Cut& ct = m.best[w];
        Lut L;
        L.wire = w;
        L.nin = ct.n;
        for (int i = 0; i < K; i++) L.in[i] = i < ct.n ? ct.l[i] : ct.l[0];
        L.tt = cone.tt(c, w, ct.l, ct.n);
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

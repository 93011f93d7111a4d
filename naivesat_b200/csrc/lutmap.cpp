// lutmap.cpp -- priority-cut 3-LUT mapping with area flow and exact-area recovery.
//
// Cuts carry the truth table of their node over their leaves (64 rows, up to
// six leaves) and are reduced to the support of that function: a cone whose
// structure has four, five or six leaves often computes a function of three
// or fewer of them (the gates of a random DAG reconverge within a few
// levels), and then it is one LUT.  Cuts wider than three leaves are kept
// only as steps towards such cones.  On the 3000-gate random DAGs of the
// benchmark configurations this covers the live gates with about 30 % fewer
// LUTs than structural 3-cuts.
#include "lutmap.h"

#include <algorithm>
#include <cmath>

namespace nsat {

namespace {

constexpr int K = 3;          // LUT inputs (lop3)
constexpr int KE = 6;         // most leaves of a cut enumerated (reduced to its function's support)
constexpr int P = 10;         // implementable cuts (<= K leaves) kept per node
constexpr int Q = 8;          // wider cuts kept per node, only as steps towards larger cones

// truth tables over up to 6 leaves: row r has leaf i = bit i of r
typedef uint64_t TT;
constexpr TT kVar[6] = {0xAAAAAAAAAAAAAAAAull, 0xCCCCCCCCCCCCCCCCull, 0xF0F0F0F0F0F0F0F0ull,
                        0xFF00FF00FF00FF00ull, 0xFFFF0000FFFF0000ull, 0xFFFFFFFF00000000ull};

struct Cut {
    uint8_t n = 0;
    uint32_t l[KE];
    uint32_t sig = 0;   // OR of 1 << (leaf % 32): more than KE bits set means more than KE leaves
    TT tt = 0;          // function of the node over the leaves
    float af = 0;
    bool operator==(const Cut& o) const {
        if (n != o.n) return false;
        for (int i = 0; i < n; i++) if (l[i] != o.l[i]) return false;
        return true;
    }
};

// merge two sorted leaf sets; false if more than `ke` leaves
bool merge(const Cut& a, const Cut& b, Cut* out, int ke) {
    int i = 0, j = 0, k = 0;
    while (i < a.n || j < b.n) {
        uint32_t v;
        if (j >= b.n || (i < a.n && a.l[i] < b.l[j])) v = a.l[i++];
        else if (i >= a.n || b.l[j] < a.l[i]) v = b.l[j++];
        else { v = a.l[i]; i++; j++; }
        if (k == ke) return false;
        out->l[k++] = v;
    }
    out->n = (uint8_t)k;
    out->sig = a.sig | b.sig;
    return true;
}

inline TT gate_eval64(uint8_t f, TT a, TT b) {
    switch (f) {
    case AND: return a & b;
    case NOR: return ~(a | b);
    case NIMPL: return a & ~b;
    default: return a ^ b;
    }
}

// exchanges variables i < j of a table
inline TT swap_vars(TT t, int i, int j) {
    const int sh = (1 << j) - (1 << i);
    const TT mi = kVar[i] & ~kVar[j], mj = ~kVar[i] & kVar[j];
    return (t & ~(mi | mj)) | ((t & mi) << sh) | ((t & mj) >> sh);
}

// x's truth table re-expressed over the leaves of `to` (a superset of x's):
// x's variable i moves to the position of its leaf in `to`, highest first,
// so every move lands on a variable x does not use
TT expand_tt(const Cut& x, const Cut& to) {
    int pos[KE];
    for (int i = 0, j = 0; i < x.n; i++) {
        while (to.l[j] != x.l[i]) j++;
        pos[i] = j;
    }
    TT t = x.tt;
    for (int i = x.n - 1; i >= 0; i--)
        if (pos[i] != i) t = swap_vars(t, i, pos[i]);
    return t;
}

// drops the leaves the function does not depend on: such a variable is
// moved up past the others and the leaf count shrinks (the table is
// independent of the variables at and above the leaf count)
void minimize(Cut* c) {
    for (int i = c->n - 1; i >= 0; i--) {
        const TT v = kVar[i];
        if (((c->tt & v) >> (1 << i)) != (c->tt & ~v)) continue;
        for (int k = i; k + 1 < c->n; k++) {
            c->tt = swap_vars(c->tt, k, k + 1);
            c->l[k] = c->l[k + 1];
        }
        c->n--;
    }
    c->sig = 0;
    for (int i = 0; i < c->n; i++) c->sig |= 1u << (c->l[i] & 31u);
}

struct Mapper {
    const Circuit& c;
    uint32_t n, W;
    std::vector<uint8_t> live;
    std::vector<uint32_t> fanout;
    std::vector<Cut> cuts;      // gate w's kept cuts: cuts[(w - n) * P .. + ncut[w - n])
    std::vector<uint8_t> ncut;
    std::vector<Cut> wide;      // gate w's kept cuts of KE leaves (not LUTs themselves)
    std::vector<uint8_t> nwide;
    std::vector<Cut> best;
    std::vector<float> af;
    std::vector<int32_t> refs;
    std::vector<uint32_t> stk;  // work list of ref_cut / deref_cut
    std::vector<uint32_t> log;  // reference increments made by ref_cut_bounded

    int ke = KE;                // leaves of the cuts enumerated (K .. KE)

    explicit Mapper(const Circuit& cc) : c(cc), n(cc.n), W(cc.wires()) {}

    // The per-node arrays live in buffers kept per host thread between
    // calls: a fresh allocation of several hundred KB per mapping costs more
    // in page faults than the mapping of a small circuit itself.
    struct Buffers {
        std::vector<uint8_t> live, ncut, nwide;
        std::vector<uint32_t> fanout;
        std::vector<Cut> cuts, wide, best;
        std::vector<float> af;
        std::vector<int32_t> refs;
    };
    void swap_buffers(Buffers& b) {
        live.swap(b.live); ncut.swap(b.ncut); nwide.swap(b.nwide); fanout.swap(b.fanout);
        cuts.swap(b.cuts); wide.swap(b.wide); best.swap(b.best); af.swap(b.af); refs.swap(b.refs);
    }

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

    // A fanin's cuts: its trivial cut first, then its kept cuts (wide ones included).
    int fanin_cuts(uint32_t x, Cut* v) const {
        int k = 0;
        Cut& triv = v[k++];
        triv.n = 1;
        triv.l[0] = x;
        triv.sig = 1u << (x & 31u);
        triv.tt = kVar[0];
        triv.af = is_gate(x) ? af[x] : 0.f;
        if (is_gate(x)) {
            const Cut* cx = cuts_of(x);
            for (int i = 0; i < ncut[x - n]; i++)
                if (!(cx[i].n == 1 && cx[i].l[0] == x)) v[k++] = cx[i];
            const Cut* wx = &wide[(size_t)(x - n) * Q];
            for (int i = 0; i < nwide[x - n]; i++) v[k++] = wx[i];
        }
        return k;
    }

    static void insert(Cut* keep, int* nk, int cap, const Cut& x) {
        int pos = *nk;
        while (pos > 0 && (x.af < keep[pos - 1].af || (x.af == keep[pos - 1].af && x.n < keep[pos - 1].n))) pos--;
        if (pos >= cap) return;
        for (int k = std::min(*nk, cap - 1); k > pos; k--) keep[k] = keep[k - 1];
        keep[pos] = x;
        if (*nk < cap) (*nk)++;
    }

    void enumerate() {
        cuts.assign((size_t)(W - n) * P, Cut());
        ncut.assign(W - n, 0);
        if (ke > K) wide.assign((size_t)(W - n) * Q, Cut());   // no wider cuts to keep at K leaves
        nwide.assign(W - n, 0);
        best.assign(W, Cut());
        af.assign(W, 0.f);
        Cut ca[P + Q + 1], cb[P + Q + 1], cand[(P + Q + 1) * (P + Q + 1)];
        constexpr uint32_t kHash = 1024;     // > 2 x the candidates of a gate
        static_assert((P + Q + 1) * (P + Q + 1) * 2 <= (int)kHash, "candidate hash size");
        std::vector<uint32_t> hstamp(kHash, 0);
        std::vector<uint16_t> hslot(kHash, 0);
        for (uint32_t w = n; w < W; w++) {
            if (!live[w]) continue;
            const Gate& g = gate(w);
            const int na = fanin_cuts(g.i0, ca), nb = fanin_cuts(g.i1, cb);
            int nc = 0;
            for (int ia = 0; ia < na; ia++)
                for (int ib = 0; ib < nb; ib++) {
                    Cut m;
                    if (__builtin_popcount(ca[ia].sig | cb[ib].sig) > ke) continue;
                    if (!merge(ca[ia], cb[ib], &m, ke)) continue;
                    m.tt = gate_eval64(g.func, expand_tt(ca[ia], m), expand_tt(cb[ib], m));
                    minimize(&m);
                    // the same leaves give the same function: keep the first
                    uint32_t h = 0x9E3779B9u * (m.n + 1);
                    for (int i = 0; i < m.n; i++) h = (h ^ m.l[i]) * 0x85EBCA6Bu;
                    h = (h ^ (h >> 15)) & (kHash - 1);
                    bool dup = false;
                    while (hstamp[h] == w) {
                        if (cand[hslot[h]] == m) { dup = true; break; }
                        h = (h + 1) & (kHash - 1);
                    }
                    if (dup) continue;
                    hstamp[h] = w;
                    hslot[h] = (uint16_t)nc;
                    float a = 1.f;
                    for (int i = 0; i < m.n; i++) {
                        uint32_t l = m.l[i];
                        if (is_gate(l)) a += af[l] / (float)std::max<uint32_t>(1, fanout[l]);
                    }
                    m.af = a;
                    cand[nc++] = m;
                }
            Cut* keep = &cuts[(size_t)(w - n) * P];
            Cut* kw = &wide[(size_t)(w - n) * Q];
            int nk = 0, nw = 0;
            for (int j = 0; j < nc; j++) {
                if (cand[j].n <= K) insert(keep, &nk, P, cand[j]);
                else insert(kw, &nw, Q, cand[j]);
            }
            ncut[w - n] = (uint8_t)nk;
            nwide[w - n] = (uint8_t)nw;
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

uint32_t live_gate_count(const Circuit& c, const std::vector<uint32_t>& which) {
    const uint32_t n = c.n, W = c.wires();
    std::vector<uint8_t> live(W, 0);
    for (uint32_t j : which) live[c.outputs[j].wire] = 1;
    uint32_t k = 0;
    for (int64_t w = (int64_t)W - 1; w >= (int64_t)n; w--) {
        if (!live[w]) continue;
        const Gate& g = c.gates[(size_t)w - n];
        live[g.i0] = live[g.i1] = 1;
        k++;
    }
    return k;
}

LutNet map_luts(const Circuit& c, const std::vector<uint32_t>& which, bool one_per_gate, int cut_leaves,
                int recovery_passes) {
    LutNet net;
    Mapper m(c);
    static thread_local Mapper::Buffers buffers;
    struct Keep {
        Mapper& m;
        ~Keep() { m.swap_buffers(buffers); }
    } keep{m};
    m.swap_buffers(buffers);
    m.ke = std::max(K, std::min(KE, cut_leaves));
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
        for (int pass = 0; pass < recovery_passes; pass++) {
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
        if (one_per_gate) {
            L.nin = ct.n;
            for (int i = 0; i < K; i++) L.in[i] = i < ct.n ? ct.l[i] : ct.l[0];
            L.tt = cone.tt(c, w, ct.l, ct.n);
        } else {
            // the cut's own table: leaf i is operand i (a = bit 2 of the lop3 row)
            L.nin = ct.n ? ct.n : 1;
            const uint32_t l0 = ct.n ? ct.l[0] : 0;   // a constant reads input 0 and ignores it
            if (!ct.n) need[0] = 1;
            for (int i = 0; i < K; i++) L.in[i] = i < ct.n ? ct.l[i] : l0;
            uint8_t t = 0;
            for (int r = 0; r < 8; r++) {
                const int a = (r >> 2) & 1, b = (r >> 1) & 1, cc = r & 1;
                int s = 0;
                if (ct.n > 0) s |= a;
                if (ct.n > 1) s |= b << 1;
                if (ct.n > 2) s |= cc << 2;
                if ((ct.tt >> s) & 1) t |= (uint8_t)(1u << r);
            }
            L.tt = t;
        }
        net.luts.push_back(L);
    }
    for (uint32_t i = 0; i < n; i++) if (need[i]) net.used_inputs.push_back(i);
    for (uint32_t j : which) net.outs.push_back(c.outputs[j]);
    return net;
}

LutNet map_luts_for(const Circuit& c, const std::vector<uint32_t>& which, bool one_per_gate, double log2_space,
                    double lut_words_per_s, bool shared_device) {
    if (one_per_gate) return map_luts(c, which, true, 3);
    // measured on the 3000-gate random DAGs of seeds 1-3: mapping time per
    // gate, and LUTs relative to three leaves, for 3..6 leaves
    static const double map_s_per_gate[4] = {1.0e-6, 2.7e-6, 5.5e-6, 9.0e-6};
    static const double ratio[4] = {1.0, 0.985, 0.965, 0.95};
    const double words = std::ldexp(1.0, (int)std::max(0.0, log2_space - 5.0));
    const double gate_search_s = words * (double)live_gate_count(c, which) / lut_words_per_s;
    if (!shared_device && gate_search_s < 0.25 * map_s_per_gate[0] * (double)c.gates.size())
        return map_luts(c, which, true, 3);
    // The second exact-area pass costs 20-35 % of the mapping and saved at
    // most one LUT on the benchmark circuits: it runs only for searches of
    // 0.1 s and more (estimated from the live gates at 0.6 LUTs per gate),
    // where its cost stays under about 1 % of the solve.
    const int passes = 0.6 * gate_search_s >= 0.1 ? 2 : 1;
    LutNet net = map_luts(c, which, false, 3, passes);
    const double search_s = words * (double)net.luts.size() / lut_words_per_s;
    int best = 3;
    double best_s = search_s;
    for (int ke = 4; ke <= KE; ke++) {
        const double t = map_s_per_gate[ke - 3] * (double)c.gates.size() + search_s * ratio[ke - 3];
        if (t < best_s) { best_s = t; best = ke; }
    }
    return best == 3 ? net : map_luts(c, which, one_per_gate, best, passes);
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

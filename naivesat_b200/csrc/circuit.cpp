// circuit.cpp -- circuit validation, hashing and gatesim text I/O.
#include "circuit.h"

#include <cctype>
#include <cstring>
#include <map>

namespace nsat {

std::string Circuit::validate() const {
    if (n == 0) return "circuit has no inputs";
    if (n > 128) return "more than 128 inputs";
    for (size_t k = 0; k < gates.size(); k++) {
        const Gate& g = gates[k];
        if (g.func > 3) return "gate " + std::to_string(k) + ": bad function";
        if (g.i0 >= n + k || g.i1 >= n + k)
            return "gate " + std::to_string(k) + ": fan-in is not an earlier wire";
    }
    if (outputs.empty()) return "circuit has no outputs";
    for (size_t j = 0; j < outputs.size(); j++)
        if (outputs[j].wire >= wires()) return "output " + std::to_string(j) + ": bad wire";
    return "";
}

uint64_t Circuit::hash() const {
    uint64_t h = 1469598103934665603ull;
    auto mix = [&](uint64_t v) {
        for (int i = 0; i < 8; i++) { h ^= (v >> (8 * i)) & 0xff; h *= 1099511628211ull; }
    };
    mix(n);
    mix(gates.size());
    for (const Gate& g : gates) { mix(g.func); mix(g.i0); mix(g.i1); }
    mix(outputs.size());
    for (const Output& o : outputs) { mix(o.wire); mix(o.neg); }
    return h;
}

uint8_t gate_tt2(uint8_t func) {
    uint8_t t = 0;
    for (int r = 0; r < 4; r++) {
        uint32_t a = (r >> 1) & 1, b = r & 1;
        if (gate_eval32(func, a ? ~0u : 0u, b ? ~0u : 0u) & 1) t |= (uint8_t)(1u << r);
    }
    return t;
}

// ---------------------------------------------------------------------------
// parser

namespace {

struct Lexer {
    const std::string& s;
    size_t i = 0;
    explicit Lexer(const std::string& t) : s(t) {}
    void ws() { while (i < s.size() && std::isspace((unsigned char)s[i])) i++; }
    bool eat(char c) { ws(); if (i < s.size() && s[i] == c) { i++; return true; } return false; }
    bool peek(char c) { ws(); return i < s.size() && s[i] == c; }
    bool number(uint64_t* v) {
        ws();
        if (i >= s.size() || !std::isdigit((unsigned char)s[i])) return false;
        uint64_t x = 0;
        while (i < s.size() && std::isdigit((unsigned char)s[i])) {
            x = x * 10 + (uint64_t)(s[i] - '0');
            if (x > (1ull << 40)) return false;
            i++;
        }
        *v = x;
        return true;
    }
    std::string ident() {
        ws();
        size_t b = i;
        while (i < s.size() && std::isalpha((unsigned char)s[i])) i++;
        return s.substr(b, i - b);
    }
};

}  // namespace

bool parse_gatesim(const std::string& text, Parsed* out, std::string* err) {
    *out = Parsed();
    size_t brace = text.find('{');
    if (brace == std::string::npos) { *err = "missing '{'"; return false; }
    // quantifier prefix: letters a/e (any case), separators ignored
    std::vector<uint8_t> quants;
    for (size_t k = 0; k < brace; k++) {
        char ch = text[k];
        if (ch == 'a' || ch == 'A') quants.push_back(1);
        else if (ch == 'e' || ch == 'E') quants.push_back(0);
        else if (std::isspace((unsigned char)ch) || ch == '_' || ch == ',' || ch == ':') continue;
        else { *err = std::string("unexpected character '") + ch + "' before '{'"; return false; }
    }
    std::string body = text.substr(brace);
    Lexer L(body);
    L.eat('{');
    struct Item { bool is_gate; uint32_t input; Gate g; std::vector<std::pair<uint64_t, bool>> outs; };
    std::vector<Item> items;
    while (!L.peek('}')) {
        if (L.i >= body.size()) { *err = "unterminated '{'"; return false; }
        Item it{};
        uint64_t v;
        if (L.number(&v)) {
            it.is_gate = false;
            it.input = (uint32_t)v;
        } else {
            std::string id = L.ident();
            for (auto& ch : id) ch = (char)std::tolower((unsigned char)ch);
            uint8_t f;
            if (id == "and") f = AND;
            else if (id == "nor") f = NOR;
            else if (id == "nimpl") f = NIMPL;
            else if (id == "xor") f = XOR;
            else { *err = "unknown gate '" + id + "'"; return false; }
            uint64_t a, b;
            if (!L.eat('(') || !L.number(&a) || !L.eat(',') || !L.number(&b) || !L.eat(')')) {
                *err = "malformed gate '" + id + "'"; return false;
            }
            it.is_gate = true;
            it.g = Gate{f, (uint32_t)a, (uint32_t)b};
        }
        while (L.eat(':')) {
            uint64_t k;
            if (!L.number(&k)) { *err = "malformed output marker"; return false; }
            bool neg = false;
            if (L.i < body.size() && body[L.i] == 'n') { neg = true; L.i++; }
            it.outs.push_back({k, neg});
        }
        items.push_back(std::move(it));
    }
    L.eat('}');
    uint64_t n;
    if (!L.eat('(') || !L.number(&n) || !L.eat(')')) { *err = "missing '(input_len)'"; return false; }
    L.ws();
    if (L.i != body.size()) { *err = "trailing text after circuit"; return false; }
    if (n == 0 || n > 128) { *err = "input_len out of range"; return false; }
    Circuit& c = out->circuit;
    c.n = (uint32_t)n;
    std::map<uint64_t, Output> outmap;
    uint32_t next_gate = c.n;
    for (const Item& it : items) {
        uint32_t wire;
        if (it.is_gate) {
            wire = next_gate++;
            c.gates.push_back(it.g);
        } else {
            if (it.input >= c.n) { *err = "input index out of range"; return false; }
            wire = it.input;
        }
        for (auto& o : it.outs) {
            if (outmap.count(o.first)) { *err = "duplicate output index"; return false; }
            outmap[o.first] = Output{wire, o.second};
        }
    }
    uint64_t expect = 0;
    for (auto& kv : outmap) {
        if (kv.first != expect++) { *err = "output indices are not contiguous from 0"; return false; }
        c.outputs.push_back(kv.second);
    }
    std::string v = c.validate();
    if (!v.empty()) { *err = v; return false; }
    if (!quants.empty() && quants.size() != c.n) { *err = "quantifier count differs from input_len"; return false; }
    out->quants = std::move(quants);
    return true;
}

std::string format_gatesim(const Circuit& c, const std::vector<uint8_t>* quants) {
    std::string s;
    if (quants && !quants->empty()) {
        for (uint8_t q : *quants) s += q ? 'a' : 'e';
        s += ' ';
    }
    std::vector<std::vector<std::pair<uint32_t, bool>>> marks(c.wires());
    for (uint32_t j = 0; j < c.outputs.size(); j++)
        marks[c.outputs[j].wire].push_back({j, c.outputs[j].neg});
    auto put_marks = [&](uint32_t w) {
        for (auto& m : marks[w]) {
            s += ':';
            s += std::to_string(m.first);
            if (m.second) s += 'n';
        }
    };
    static const char* names[4] = {"and", "nor", "nimpl", "xor"};
    s += '{';
    for (uint32_t i = 0; i < c.n; i++) {
        s += std::to_string(i);
        put_marks(i);
        s += ' ';
    }
    for (uint32_t k = 0; k < c.gates.size(); k++) {
        const Gate& g = c.gates[k];
        s += names[g.func];
        s += '(' + std::to_string(g.i0) + ',' + std::to_string(g.i1) + ')';
        put_marks(c.n + k);
        if (k + 1 < c.gates.size()) s += ' ';
    }
    s += "}(" + std::to_string(c.n) + ")";
    return s;
}

}  // namespace nsat

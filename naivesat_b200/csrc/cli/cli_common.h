// cli_common.h -- shared pieces of the four command-line tools: argument
// parsing in the style of the reference's clap definitions, circuit loading
// through the C ABI, scalar replay for the witness checks, and number
// formatting identical to the reference's println! formats.
#pragma once
#include <nsat.h>

#include <chrono>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>
#include <string>
#include <vector>

namespace cli {

typedef unsigned __int128 u128;

[[noreturn]] inline void die(const std::string& msg, int code = 2) {
    fprintf(stderr, "error: %s\n", msg.c_str());
    exit(code);
}

// Minimal clap-like parser: positional arguments in order, flags by short or
// long name, values as the next argument or after '='.
struct Args {
    struct Opt { std::string shrt, lng; bool takes_value; std::string help; };
    std::vector<Opt> opts;
    std::vector<std::string> positional_names;
    std::map<std::string, std::string> values;   // by long name
    std::vector<std::string> positional;
    std::string prog, about;

    void flag(const char* s, const char* l, const char* help) { opts.push_back({s, l, false, help}); }
    void option(const char* s, const char* l, const char* help) { opts.push_back({s, l, true, help}); }
    void pos(const char* name) { positional_names.push_back(name); }

    void usage(FILE* f) const {
        fprintf(f, "%s\n\nUsage: %s [OPTIONS]", about.c_str(), prog.c_str());
        for (auto& p : positional_names) fprintf(f, " <%s>", p.c_str());
        fprintf(f, "\n\nOptions:\n");
        for (auto& o : opts)
            fprintf(f, "  %s%s--%s%s  %s\n", o.shrt.empty() ? "" : ("-" + o.shrt).c_str(),
                    o.shrt.empty() ? "" : ", ", o.lng.c_str(), o.takes_value ? " <VALUE>" : "", o.help.c_str());
        fprintf(f, "  -h, --help  Print help\n");
    }

    void parse(int argc, char** argv) {
        prog = argv[0];
        for (int i = 1; i < argc; i++) {
            std::string a = argv[i];
            if (a == "-h" || a == "--help") { usage(stdout); exit(0); }
            if (a.size() > 1 && a[0] == '-' && !(a.size() > 1 && isdigit((unsigned char)a[1]))) {
                std::string name, val;
                bool has_val = false;
                const Opt* o = nullptr;
                if (a.rfind("--", 0) == 0) {
                    name = a.substr(2);
                    size_t eq = name.find('=');
                    if (eq != std::string::npos) { val = name.substr(eq + 1); name = name.substr(0, eq); has_val = true; }
                    for (auto& x : opts) if (x.lng == name) o = &x;
                } else {
                    name = a.substr(1, 1);
                    if (a.size() > 2) { val = a.substr(2); has_val = true; }
                    for (auto& x : opts) if (x.shrt == name) o = &x;
                }
                if (!o) { usage(stderr); die("unexpected argument '" + a + "'"); }
                if (o->takes_value) {
                    if (!has_val) {
                        if (i + 1 >= argc) die("a value is required for '--" + o->lng + "'");
                        val = argv[++i];
                    }
                    values[o->lng] = val;
                } else {
                    values[o->lng] = "1";
                }
            } else {
                positional.push_back(a);
            }
        }
        if (positional.size() != positional_names.size()) {
            usage(stderr);
            die("expected " + std::to_string(positional_names.size()) + " positional argument(s)");
        }
    }
    bool has(const char* lng) const { return values.count(lng) != 0; }
    std::string get(const char* lng, const std::string& def = "") const {
        auto it = values.find(lng);
        return it == values.end() ? def : it->second;
    }
    uint64_t num(const char* lng, uint64_t def) const {
        auto it = values.find(lng);
        if (it == values.end()) return def;
        char* end = nullptr;
        unsigned long long v = strtoull(it->second.c_str(), &end, 10);
        if (!end || *end) die("invalid number for --" + std::string(lng) + ": " + it->second);
        return v;
    }
};

inline std::string read_file(const std::string& path) {
    std::ifstream f(path, std::ios::binary);
    if (!f) die("cannot read " + path, 1);
    std::ostringstream s;
    s << f.rdbuf();
    return s.str();
}

// Owns a parsed circuit (gatesim text) and its flat arrays.
struct Loaded {
    nsat_parsed* p = nullptr;
    nsat_circuit_desc d{};
    const uint8_t* quants = nullptr;
    ~Loaded() { if (p) nsat_parsed_free(p); }
};

inline void load_circuit(const std::string& path, Loaded* L) {
    std::string text = read_file(path);
    if (nsat_parse(text.data(), text.size(), &L->p) != NSAT_OK) die("cannot parse circuit " + path, 1);
    nsat_parsed_get(L->p, &L->d, &L->quants);
}

// Execution type strings of the reference (main.rs:26-50); every form maps to
// CUDA devices: "cpu" and "opencl:N" to one device (0 / N), the combined
// forms to all visible devices (cpu_and_opencl_1[d]:N to device N).
struct ExecType {
    std::vector<int> devices;
    std::string label;
};

inline ExecType parse_exec_type(const std::string& s) {
    ExecType e;
    int ndev = nsat_device_count();
    auto num_after = [&](size_t pos) {
        char* end = nullptr;
        long v = strtol(s.c_str() + pos, &end, 10);
        if (!end || *end || v < 0) die("Unknown exec type");
        return (int)v;
    };
    if (s == "cpu") { e.devices = {0}; e.label = "CUDA device=0 (for -t cpu)"; }
    else if (s.rfind("opencl:", 0) == 0) { int d = num_after(7); e.devices = {d}; e.label = "CUDA device=" + std::to_string(d); }
    else if (s == "cpu_and_opencl" || s == "cpu_and_opencl_d") {
        for (int i = 0; i < ndev; i++) e.devices.push_back(i);
        e.label = "all CUDA devices (" + std::to_string(ndev) + ")";
    } else if (s.rfind("cpu_and_opencl_1d:", 0) == 0) { int d = num_after(18); e.devices = {d}; e.label = "CUDA device=" + std::to_string(d); }
    else if (s.rfind("cpu_and_opencl_1:", 0) == 0) { int d = num_after(17); e.devices = {d}; e.label = "CUDA device=" + std::to_string(d); }
    else die("Unknown exec type");
    if (e.devices.empty()) die("no CUDA device", 1);
    for (int d : e.devices) if (d >= ndev) die("CUDA device " + std::to_string(d) + " not present", 1);
    return e;
}

// Scalar evaluation of a circuit, used to re-verify witnesses the way the
// reference does with circuit.eval (main.rs:373-381, greedysatostop.rs:1114).
inline std::vector<uint8_t> eval_scalar(const nsat_circuit_desc& d, const std::vector<uint8_t>& in) {
    std::vector<uint8_t> w(d.input_len + d.gate_num);
    for (uint32_t i = 0; i < d.input_len; i++) w[i] = in[i] & 1;
    for (uint32_t k = 0; k < d.gate_num; k++) {
        uint8_t a = w[d.gates[3 * k + 1]], b = w[d.gates[3 * k + 2]];
        uint8_t v;
        switch (d.gates[3 * k]) {
        case NSAT_AND: v = a & b; break;
        case NSAT_NOR: v = !(a | b); break;
        case NSAT_NIMPL: v = a & !b; break;
        default: v = a ^ b; break;
        }
        w[d.input_len + k] = v;
    }
    std::vector<uint8_t> out(d.output_num);
    for (uint32_t j = 0; j < d.output_num; j++) out[j] = w[d.outputs[2 * j]] ^ (d.outputs[2 * j + 1] & 1);
    return out;
}

// {:0width$b}
inline std::string binary(u128 v, uint32_t width) {
    std::string s;
    for (int b = (int)width - 1; b >= 0; b--) s += ((v >> b) & 1) ? '1' : '0';
    if (width == 0) s = "0";
    return s;
}

inline std::string decimal(u128 v) {
    if (v == 0) return "0";
    std::string s;
    while (v) { s.insert(s.begin(), (char)('0' + (int)(v % 10))); v /= 10; }
    return s;
}

// {:0width$}
inline std::string decimal_padded(u128 v, size_t width) {
    std::string s = decimal(v);
    while (s.size() < width) s.insert(s.begin(), '0');
    return s;
}

inline double now_s() {
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

inline nsat_ctx* open_ctx(int device, const Args& a) {
    nsat_opts o{};
    o.block_threads = (uint32_t)a.num("opencl-group-len", 0);
    o.no_optimize = a.has("no-optimize-negs") ? 1 : 0;
    o.verbose = getenv("NSAT_VERBOSE") ? 1 : 0;
    nsat_ctx* ctx = nullptr;
    int rc = nsat_create(device, &o, &ctx);
    if (rc != NSAT_OK) die(std::string("nsat_create: ") + nsat_strerror(rc), 1);
    return ctx;
}

// With NSAT_AUTOTUNE set in the environment, the circuit's launch shape is
// tuned before solving (nsat_autotune, remembered in the kernel cache
// directory, so the cost is paid once per circuit and GPU).  Answers do not
// depend on it.
inline int maybe_autotune(nsat_ctx* ctx, nsat_circuit* c, uint32_t kind, const uint8_t* quants) {
    if (!getenv("NSAT_AUTOTUNE")) return NSAT_OK;
    nsat_tune_opts o{};
    o.kind = kind;
    o.persist = 1;
    o.quants = quants;
    nsat_tune_result r{};
    const int rc = nsat_autotune(ctx, c, &o, &r);
    if (rc == NSAT_OK && getenv("NSAT_VERBOSE"))
        fprintf(stderr, "[nsat] autotune: %u threads, %u CTAs/SM, %u CTA bits (%s, %.2fx)\n", r.block_threads,
                r.min_blocks, r.cta_bits_max, r.from_cache ? "cached" : "measured",
                r.default_rate > 0 ? r.best_rate / r.default_rate : 0.0);
    return rc;
}

inline void check(nsat_ctx* ctx, int rc, const char* what) {
    if (rc != NSAT_OK) die(std::string(what) + ": " + nsat_strerror(rc) + " " + nsat_last_error(ctx), 1);
}

}  // namespace cli

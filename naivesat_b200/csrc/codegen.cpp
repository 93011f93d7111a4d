// codegen.cpp -- emit the per-circuit CUDA source compiled by NVRTC.
#include "codegen.h"

#include <cstdio>
#include <sstream>

namespace nsat {

std::string KernelConfig::key() const {
    std::ostringstream s;
    s << "mode=" << (int)mode << " nin=" << nin << " nb=" << nb << " c=" << c << " it=" << it << " wb=" << wb << " cb=" << cb
      << " m=" << m << " q0all=" << q0all << " allbits=" << allbits << " data=" << data
      << " fmt=" << fmt << " nout=" << nout << " minb=" << minb << " sync=" << sync_every << " map=";
    for (int v : in_of_bit) s << v << ',';
    return s.str();
}

namespace {

const char* kPrelude = R"NSAT(
typedef unsigned int u32;
typedef unsigned long long u64;
)NSAT";

const uint32_t kLanePat[5] = {0xAAAAAAAAu, 0xCCCCCCCCu, 0xF0F0F0F0u, 0xFF00FF00u, 0xFFFF0000u};

// sync_every > 0: a CTA barrier after every sync_every LUTs, so the CTA's
// warps walk the evaluation code together and share instruction-cache lines
// (the unrolled evaluation of a large circuit is larger than the
// instruction cache; c1 at 64: ALU pipe 89 % -> 0.99 of the lop3 peak).  Only
// for kernels whose every thread runs the same number of evaluations.
void emit_luts(std::ostringstream& s, const LutNet& net, uint32_t sync_every = 0) {
    for (uint32_t i : net.used_inputs) s << "    const u32 w" << i << " = x[" << i << "];\n";
    uint32_t k = 0;
    // one lop3.b32 per LUT, the truth table as its immediate; written as
    // inline asm in place (a helper template per call site costs NVVM about
    // twice the compile time on circuits of a few thousand gates).  The lines
    // are appended directly: the LUTs are most of the source, and formatting
    // them through printf took most of the generation time.
    static const char kHex[] = "0123456789abcdef";
    auto dec = [](std::string& o, uint32_t v) {
        char t[10];
        int d = 0;
        do { t[d++] = (char)('0' + v % 10); v /= 10; } while (v);
        while (d) o.push_back(t[--d]);
    };
    std::string b;
    b.reserve(net.luts.size() * 112 + (sync_every ? net.luts.size() / sync_every * 20 : 0) + 16);
    for (const Lut& L : net.luts) {
        b += "    u32 w";
        dec(b, L.wire);
        b += "; asm(\"lop3.b32 %0, %1, %2, %3, 0x";
        b.push_back(kHex[L.tt >> 4]);
        b.push_back(kHex[L.tt & 15]);
        b += ";\" : \"=r\"(w";
        dec(b, L.wire);
        b += ") : \"r\"(w";
        dec(b, L.in[0]);
        b += "), \"r\"(w";
        dec(b, L.in[1]);
        b += "), \"r\"(w";
        dec(b, L.in[2]);
        b += "));\n";
        if (sync_every && ++k % sync_every == 0) b += "    __syncthreads();\n";
    }
    s.write(b.data(), (std::streamsize)b.size());
}

}  // namespace

std::string generate_source(const KernelConfig& kc, const LutNet& net) {
    std::ostringstream s;
    s << "// generated: " << kc.key() << "\n";
    s << kPrelude;
    s << "#define NSAT_MODE_SAT " << (kc.mode == Mode::SAT ? 1 : 0) << "\n";
    s << "#define NSAT_MODE_QSAT " << (kc.mode == Mode::QSAT ? 1 : 0) << "\n";
    s << "#define NSAT_MODE_TABLE " << (kc.mode == Mode::TABLE ? 1 : 0) << "\n";
    s << "#define NSAT_DATA " << (kc.data ? 1 : 0) << "\n";
    s << "#define NSAT_FMT " << kc.fmt << "\n";
    s << "constexpr int NSAT_NIN = " << kc.nin << ";\n";
    s << "constexpr int NSAT_NOUT = " << kc.nout << ";\n";
    s << "constexpr int NSAT_NB = " << kc.nb << ";\n";
    s << "constexpr int NSAT_NT = " << kc.threads() << ";\n";
    if (kc.minb) s << "#define NSAT_BOUNDS __launch_bounds__(" << kc.threads() << ", " << kc.minb << ")\n";
    else s << "#define NSAT_BOUNDS __launch_bounds__(" << kc.threads() << ")\n";
    s << "constexpr int NSAT_IT = " << kc.it << ";\n";
    s << "constexpr int NSAT_WB = " << kc.wb << ";\n";
    s << "constexpr int NSAT_CB = " << kc.cb << ";\n";
    s << "constexpr int NSAT_C = " << kc.c << ";\n";
    s << "constexpr int NSAT_M = " << kc.m << ";\n";
    s << "constexpr int NSAT_Q0ALL = " << (kc.q0all ? 1 : 0) << ";\n";
    s << "constexpr u64 NSAT_ALLBITS = " << kc.allbits << "ull;\n";

    // enumeration: which circuit input each bit drives
    const uint32_t it_lo = 10, wb_lo = 10 + kc.it, cb_lo = wb_lo + kc.wb, c_lo = cb_lo + kc.cb;
    std::ostringstream fixed, iter, word;
    char buf[160];
    for (uint32_t p = 0; p < kc.nb; p++) {
        int in = kc.in_of_bit[p];
        if (in < 0) continue;
        if (p < 5) {
            snprintf(buf, sizeof(buf), "    x[%d] = 0x%08xu;\n", in, kLanePat[p]);
            fixed << buf;
            word << buf;
            continue;
        }
        snprintf(buf, sizeof(buf), "    x[%d] = 0u - (u32)((w >> %u) & 1ull);\n", in, p - 5);
        word << buf;
        if (p < it_lo) snprintf(buf, sizeof(buf), "    x[%d] = 0u - ((lane >> %u) & 1u);\n", in, p - 5);
        else if (p < wb_lo) {
            snprintf(buf, sizeof(buf), "    x[%d] = 0u - ((it >> %u) & 1u);\n", in, p - it_lo);
            iter << buf;
            continue;
        } else if (p < cb_lo) snprintf(buf, sizeof(buf), "    x[%d] = 0u - ((warp >> %u) & 1u);\n", in, p - wb_lo);
        else if (p < c_lo) snprintf(buf, sizeof(buf), "    x[%d] = 0u - ((cta >> %u) & 1u);\n", in, p - cb_lo);
        else if (p - c_lo < 64) snprintf(buf, sizeof(buf), "    x[%d] = 0u - (u32)((launch >> %u) & 1ull);\n", in, p - c_lo);
        else snprintf(buf, sizeof(buf), "    x[%d] = 0u;\n", in);
        fixed << buf;
    }
    s << "__device__ __forceinline__ void nsat_inputs_fixed(u32* x, u32 lane, u32 warp, u32 cta, u64 launch) {\n"
      << "    (void)lane; (void)warp; (void)cta; (void)launch;\n"
      << fixed.str() << "}\n";
    s << "__device__ __forceinline__ void nsat_inputs_iter(u32* x, u32 it) {\n    (void)it;\n"
      << iter.str() << "}\n";
    s << "__device__ __forceinline__ void nsat_inputs_word(u32* x, u64 w) {\n    (void)w;\n"
      << word.str() << "}\n";

    // circuit evaluation
    if (kc.mode == Mode::TABLE) {
        s << "__device__ __forceinline__ void nsat_eval1(const u32* x) {}\n";
        s << "__device__ __forceinline__ void nsat_eval_all(const u32* x, u32* o) {\n";
        emit_luts(s, net);
        for (size_t j = 0; j < net.outs.size(); j++)
            s << "    o[" << j << "] = " << (net.outs[j].neg ? "~" : "") << "w" << net.outs[j].wire << ";\n";
        s << "}\n";
    } else {
        s << "__device__ __forceinline__ u32 nsat_eval1(const u32* x) {\n";
        if (!kc.data) {
            // the SAT and QSAT kernels run the same number of evaluations in
            // every thread of a CTA, so barriers inside the evaluation are safe
            const bool uniform = kc.mode == Mode::SAT || kc.mode == Mode::QSAT;
            emit_luts(s, net, uniform && kc.threads() > 32 ? kc.sync_every : 0);
            s << "    return " << (net.outs[0].neg ? "~" : "") << "w" << net.outs[0].wire << ";\n";
        } else {
            s << "    return 0u;\n";
        }
        s << "}\n";
        s << "__device__ __forceinline__ void nsat_eval_all(const u32* x, u32* o) {}\n";
    }
    s << kDeviceTemplate;
    return s.str();
}

}  // namespace nsat

// nsat_api.cpp -- the C ABI (include/nsat.h): contexts, circuits, and the SAT,
// QSAT and SATOSTOP drivers around the NVRTC-specialised sm_100a kernels.
#include "nsat.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <functional>
#include <atomic>
#include <thread>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "circuit.h"
#include "codegen.h"
#include "jit.h"
#include "lutmap.h"
#include "qreducer.h"
#include "internal.h"
#include "static_kernels.h"

using namespace nsat;
typedef unsigned __int128 u128;

namespace {

// Must match struct LaunchOut in device_template.cuh.
struct LaunchOut {
    uint64_t min_idx;
    uint64_t count;
    uint32_t tree;
    uint32_t ticket;
    uint32_t any;
    uint32_t err;
};
static_assert(sizeof(LaunchOut) == 32, "LaunchOut layout");

constexpr int kRing = 4;   // launches in flight before the host reads results

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

}  // namespace

struct nsat_ctx {
    int device = 0;
    nsat_opts opts{};
    cudaStream_t stream = nullptr;
    int sm_count = 0;
    std::string last_err;
    LaunchOut* d_out = nullptr;       // kRing slots
    LaunchOut* h_out = nullptr;       // pinned mirror
    LaunchOut* h_init = nullptr;      // pinned init template
    cudaEvent_t ev0[kRing]{}, ev1[kRing]{}, evd[kRing]{};
    unsigned char* d_scratch = nullptr;
    size_t scratch_bytes = 0;
    uint32_t* d_data = nullptr;
    size_t data_bytes = 0;
    NsatJoinState* d_join = nullptr;
    NsatJoinState* h_join = nullptr;
    // loaded kernels by everything their generated source depends on (the
    // kernel configuration, the entry point and the LUT net, compared
    // whole): a fresh circuit handle whose cover and launch configuration
    // were seen before skips generating and hashing the source.  The entries
    // are weak, so the JIT module cache alone decides what stays loaded.
    std::unordered_map<std::string, std::pair<CUfunction, std::weak_ptr<JitModule>>> by_inputs;
    cudaMemPool_t pool = nullptr;     // per-call buffers (ctx_alloc)
};

// Memory the context's pool keeps for reuse after its buffers are freed;
// beyond it the pool returns memory at the next synchronisation.
constexpr uint64_t kPoolKeepBytes = 8ull << 30;

// Launch shape of the evaluator kernels: threads per CTA, CTAs per SM the
// kernels are compiled for, and the cap on CTA bits per launch (the rest of
// a launch's bits are loop iterations per warp).  0 = the context's choice.
struct Shape {
    uint32_t block_threads = 0, min_blocks = 0, cb_max = 0;
    uint32_t sync_every = 0;     // 0 = default (kDefaultSync); kNoSync = no barriers
};

constexpr uint32_t kDefaultSync = 64;
constexpr uint32_t kNoSync = 0xffffffffu;

uint32_t sync_of(const Shape& sh) { return sh.sync_every == kNoSync ? 0 : (sh.sync_every ? sh.sync_every : kDefaultSync); }

struct nsat_circuit {
    nsat_ctx* ctx = nullptr;
    int device = -1;             // ctx's device (read again when the handle is freed)
    Circuit circ;
    std::map<std::string, LutNet> nets;
    // kernels loaded for this handle, by net key + kernel config + entry
    // point: a repeated solve skips generating and hashing the source
    std::map<std::string, std::pair<CUfunction, std::shared_ptr<JitModule>>> kernels;
    Shape tuned;                 // set by nsat_autotune (per kind)
    Shape tuned_qsat;
};

struct nsat_table {
    nsat_ctx* ctx = nullptr;
    uint32_t n = 0, fmt = 0;
    uint64_t N = 0;
    size_t entry_bytes = 0;
    void* buf[2] = {nullptr, nullptr};
    int cur = 0;          // buffer holding the current table
    bool any_stop = false;
    double build_ms = 0;
    ~nsat_table() {       // the buffers came from the context's pool
        if (buf[0] || buf[1]) {
            cudaSetDevice(ctx->device);
            nsat::ctx_free(ctx, buf[0]);
            nsat::ctx_free(ctx, buf[1]);
        }
    }
};

struct nsat_parsed {
    Parsed p;
    std::vector<uint32_t> gates, outputs;
};

namespace {

int fail(nsat_ctx* ctx, int code, const std::string& msg) {
    if (ctx) ctx->last_err = msg;
    return code;
}

#define CK(call)                                                                         \
    do {                                                                                 \
        cudaError_t e_ = (call);                                                         \
        if (e_ != cudaSuccess)                                                           \
            return fail(ctx, e_ == cudaErrorMemoryAllocation ? NSAT_ENOMEM : NSAT_ECUDA, \
                        std::string(#call) + ": " + cudaGetErrorString(e_));             \
    } while (0)

int set_device(nsat_ctx* ctx) {
    cudaError_t e = cudaSetDevice(ctx->device);
    if (e != cudaSuccess) return fail(ctx, NSAT_ECUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(e));
    return NSAT_OK;
}

Circuit from_desc(const nsat_circuit_desc* d) {
    Circuit c;
    c.n = d->input_len;
    c.gates.resize(d->gate_num);
    for (uint32_t k = 0; k < d->gate_num; k++)
        c.gates[k] = Gate{(uint8_t)d->gates[3 * k], d->gates[3 * k + 1], d->gates[3 * k + 2]};
    c.outputs.resize(d->output_num);
    for (uint32_t j = 0; j < d->output_num; j++)
        c.outputs[j] = Output{d->outputs[2 * j], d->outputs[2 * j + 1] != 0};
    return c;
}

std::string net_key(const nsat_circuit* c, const std::vector<uint32_t>& which) {
    std::string key = c->ctx->opts.no_optimize ? "raw:" : "lut:";
    for (uint32_t j : which) key += std::to_string(j) + ",";
    return key;
}

const LutNet& get_net(nsat_circuit* c, const std::vector<uint32_t>& which) {
    const std::string key = net_key(c, which);
    auto it = c->nets.find(key);
    if (it != c->nets.end()) return it->second;
    return c->nets[key] = map_luts_for(c->circ, which, c->ctx->opts.no_optimize != 0, c->circ.n,
                                       kCompiledLutWordsPerS);
}

// The shape a solve uses: the circuit's tuned one when set, else the
// context's options.
Shape effective_shape(const nsat_ctx* ctx, const Shape& tuned) {
    Shape s;
    s.block_threads = tuned.block_threads ? tuned.block_threads : ctx->opts.block_threads;
    s.min_blocks = tuned.block_threads ? tuned.min_blocks : ctx->opts.min_blocks;
    s.cb_max = tuned.cb_max;
    s.sync_every = tuned.sync_every;
    return s;
}

// Splits the launch's C enumeration bits into lane(5)+warp-lane(5)+IT+WB+CB.
void choose_shape(uint32_t C, uint32_t block_threads, KernelConfig* kc, uint32_t cb_max = 0) {
    uint32_t wb = 3;
    if (block_threads) {
        wb = 0;
        while ((32u << (wb + 1)) <= block_threads && wb < 5) wb++;
    }
    if (wb > C - 10) wb = C - 10;
    uint32_t rest = C - 10 - wb;
    // small launches keep 4 iterations per warp while the grid still holds
    // 2^12 warps (one wave at 24 resident warps per SM): one word per thread
    // in 2048 CTAs left c0 (2^24 assignments) launch-bound at 13.6 us, 256
    // CTAs of 8 warps latency-bound at 12.8 us, 4096 warps of 4 iterations
    // took 8.7 us
    const uint32_t cap = cb_max ? cb_max : 12;
    const uint32_t wave = wb < 12 ? 12 - wb : 0;       // CTA bits for 2^12 warps
    uint32_t cb = std::min<uint32_t>(rest, cap);
    if (rest >= 2) cb = std::min<uint32_t>(cb, rest - 2);
    cb = std::max<uint32_t>(cb, std::min<uint32_t>(rest, std::min<uint32_t>(wave, cap)));
    uint32_t it = rest - cb;
    if (it > 10) { it = 10; cb = rest - 10; }
    kc->wb = wb; kc->it = it; kc->cb = cb; kc->c = C;
}

// CTAs per SM the evaluator kernels are compiled for when the caller does
// not say: 24 warps per SM (80 registers per thread, no spills on the
// 3000-gate circuits) measured 9 % faster than the register-unbounded
// 16-warp build on c1; tiny kernels are not register limited either way.
// Circuits of at most 64 mapped lop3 (e.g. the 32-input adder QSAT) are
// bound by the reduction stages' latency, not by registers: 48 warps per SM
// measured 18 % faster than 24 there and no better elsewhere.
uint32_t default_min_blocks(const KernelConfig& kc, uint32_t lop3) {
    const uint32_t warps = 1u << kc.wb;
    const uint32_t target = (lop3 && lop3 <= 64) ? 48 : 24;
    return warps >= target ? 1 : target / warps;
}

int ensure_scratch(nsat_ctx* ctx, size_t bytes) {
    if (ctx->scratch_bytes >= bytes) return NSAT_OK;
    if (ctx->d_scratch) cudaFree(ctx->d_scratch);
    ctx->d_scratch = nullptr;
    ctx->scratch_bytes = 0;
    CK(cudaMalloc(&ctx->d_scratch, bytes));
    ctx->scratch_bytes = bytes;
    return NSAT_OK;
}

// The inputs of generate_source as one byte string: the configuration key,
// the entry point and the net's LUTs, inputs and outputs (counts first).
std::string source_inputs(const KernelConfig& kc, const LutNet& net, const char* name) {
    std::string k = kc.key();
    k += '|';
    k += name;
    k += '|';
    auto put = [&k](const void* p, size_t n) { k.append(static_cast<const char*>(p), n); };
    const uint32_t counts[3] = {(uint32_t)net.luts.size(), (uint32_t)net.used_inputs.size(),
                                (uint32_t)net.outs.size()};
    put(counts, sizeof(counts));
    k.reserve(k.size() + net.luts.size() * 18 + net.used_inputs.size() * 4 + net.outs.size() * 5);
    for (const Lut& L : net.luts) {
        put(&L.wire, 4);
        put(&L.nin, 1);
        put(L.in, 12);
        put(&L.tt, 1);
    }
    put(net.used_inputs.data(), net.used_inputs.size() * 4);
    for (const Output& o : net.outs) {
        const uint8_t neg = o.neg ? 1 : 0;
        put(&o.wire, 4);
        put(&neg, 1);
    }
    return k;
}

int get_kernel(nsat_ctx* ctx, const KernelConfig& kc, const LutNet& net, const char* name,
               CUfunction* fn, std::shared_ptr<JitModule>* holder) {
    std::string key = source_inputs(kc, net, name);
    auto it = ctx->by_inputs.find(key);
    if (it != ctx->by_inputs.end()) {
        if (std::shared_ptr<JitModule> m = it->second.second.lock()) {
            *fn = it->second.first;
            *holder = std::move(m);
            return NSAT_OK;
        }
    }
    std::string src = generate_source(kc, net);
    std::string err;
    int rc = jit_get(ctx->device, src, {name}, ctx->opts.verbose != 0, holder, &err);
    if (rc == -3) return fail(ctx, NSAT_ECOMPILE, err);
    if (rc != 0) return fail(ctx, NSAT_ECUDA, err);
    *fn = (*holder)->fns[name];
    if (ctx->by_inputs.size() >= 1024) {     // drop entries whose modules were evicted
        for (auto e = ctx->by_inputs.begin(); e != ctx->by_inputs.end();)
            e = e->second.second.expired() ? ctx->by_inputs.erase(e) : std::next(e);
        if (ctx->by_inputs.size() >= 1024) ctx->by_inputs.clear();
    }
    ctx->by_inputs[std::move(key)] = {*fn, *holder};
    return NSAT_OK;
}

// get_kernel through the circuit handle's kernel map.
int get_circuit_kernel(nsat_ctx* ctx, nsat_circuit* c, const std::vector<uint32_t>& which,
                       const KernelConfig& kc, const LutNet& net, const char* name, CUfunction* fn,
                       std::shared_ptr<JitModule>* holder) {
    const std::string key = net_key(c, which) + "|" + kc.key() + "|" + name;
    auto it = c->kernels.find(key);
    if (it != c->kernels.end()) {
        *fn = it->second.first;
        *holder = it->second.second;
        return NSAT_OK;
    }
    if (int rc = get_kernel(ctx, kc, net, name, fn, holder)) return rc;
    c->kernels[key] = {*fn, *holder};
    return NSAT_OK;
}

int launch(nsat_ctx* ctx, CUfunction fn, unsigned grid, unsigned threads, void** params) {
    std::string err;
    const DriverApi* api = driver_api(&err);
    if (!api) return fail(ctx, NSAT_ECUDA, err);
    CUresult r = api->LaunchKernel(fn, grid, 1, 1, threads, 1, 1, 0, (CUstream)ctx->stream, params, nullptr);
    if (r != CUDA_SUCCESS) {
        const char* s = nullptr;
        api->GetErrorString(r, &s);
        return fail(ctx, NSAT_ECUDA, std::string("cuLaunchKernel: ") + (s ? s : "?"));
    }
    return NSAT_OK;
}

int ctz128(u128 v) {
    if (v == 0) return 128;
    uint64_t lo = (uint64_t)v;
    if (lo) return __builtin_ctzll(lo);
    return 64 + __builtin_ctzll((uint64_t)(v >> 64));
}

uint64_t reverse_bits(uint64_t v, uint32_t bits) {
    uint64_t r = 0;
    for (uint32_t k = 0; k < bits; k++) r |= ((v >> k) & 1ull) << (bits - 1 - k);
    return r;
}

// Runs a sequence of launches of one kernel with a ring of result slots:
// `issue(k, slot)` enqueues launch k, `consume(k, out, ms)` sees its result and
// returns false to stop issuing.  Device time is the sum of the per-launch
// CUDA event intervals.
// `claim(k, slot)`, when given, is asked before launch k is prepared and
// returns false when there is nothing more to issue (a shared chunk queue ran
// out); launches already issued are still consumed.
struct ClaimAll {
    bool operator()(uint64_t, int) const { return true; }
};

template <typename Issue, typename Consume, typename Claim = ClaimAll>
int run_ring(nsat_ctx* ctx, uint64_t total, Issue issue, Consume consume, double* dev_ms,
             uint32_t* launches, Claim claim = Claim()) {
    uint64_t issued = 0, done = 0;
    bool stop = false;
    *dev_ms = 0;
    *launches = 0;
    while (done < issued || (!stop && issued < total)) {
        if (!stop && issued < total && issued - done < (uint64_t)kRing && !claim(issued, (int)(issued % kRing))) {
            stop = true;
            continue;      // nothing more to issue: consume what is in flight, if anything
        }
        if (!stop && issued < total && issued - done < (uint64_t)kRing) {
            const int slot = (int)(issued % kRing);
            CK(cudaMemcpyAsync(ctx->d_out + slot, ctx->h_init, sizeof(LaunchOut), cudaMemcpyHostToDevice,
                               ctx->stream));
            CK(cudaEventRecord(ctx->ev0[slot], ctx->stream));
            int rc = issue(issued, slot);
            if (rc) {
                // earlier launches may still be queued: finish them before the
                // caller can release the module they run from
                cudaStreamSynchronize(ctx->stream);
                return rc;
            }
            CK(cudaEventRecord(ctx->ev1[slot], ctx->stream));
            CK(cudaMemcpyAsync(ctx->h_out + slot, ctx->d_out + slot, sizeof(LaunchOut), cudaMemcpyDeviceToHost,
                               ctx->stream));
            CK(cudaEventRecord(ctx->evd[slot], ctx->stream));
            issued++;
            continue;
        }
        const int slot = (int)(done % kRing);
        CK(cudaEventSynchronize(ctx->evd[slot]));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->ev0[slot], ctx->ev1[slot]));
        *dev_ms += ms;
        (*launches)++;
        if (!stop) {
            if (!consume(done, ctx->h_out[slot])) stop = true;
        }
        done++;
    }
    return NSAT_OK;
}


// ---------------------------------------------------------------------------
// kernel plans (shared by the solvers and nsat_jit_check)

struct SatPlan {
    KernelConfig kc;
    uint32_t d = 0, C = 0;
    u128 bp = 0, ep = 0;   // range in the padded index space
};

int plan_sat(uint32_t n, const nsat_sat_opts& o, const Shape& sh, SatPlan* pl, std::string* err, uint32_t lop3 = 0) {
    const uint32_t block_threads = sh.block_threads, min_blocks = sh.min_blocks;
    const uint32_t d = n < 15 ? 15 - n : 0;     // dummy low bits for tiny circuits
    const uint32_t np = n + d;
    if (np > 128) { *err = "too many inputs"; return NSAT_EUNSUPPORTED; }
    const u128 full = (u128)1 << n;
    u128 begin = ((u128)o.begin_hi << 64) | o.begin_lo;
    u128 end = ((u128)o.end_hi << 64) | o.end_lo;
    if (end == 0) end = full;
    if (begin >= end || end > full) { *err = "bad range"; return NSAT_EINVAL; }
    const u128 bp = begin << d, ep = end << d;
    uint32_t C = o.chunk_bits ? std::max<uint32_t>(15, o.chunk_bits + d) : 34;
    C = std::min<uint32_t>(C, np);
    C = std::min<uint32_t>(C, (uint32_t)ctz128(bp));
    C = std::min<uint32_t>(C, (uint32_t)ctz128(ep - bp));
    if (C < 10) { *err = "range must be aligned to 2^10 assignments"; return NSAT_EINVAL; }
    if (np - C > 64) { *err = "more than 2^64 launches"; return NSAT_EUNSUPPORTED; }
    KernelConfig& kc = pl->kc;
    kc.mode = Mode::SAT;
    kc.nin = np;
    kc.nb = np;
    kc.in_of_bit.resize(np);
    for (uint32_t p = 0; p < np; p++) kc.in_of_bit[p] = p < d ? -1 : (int)(p - d);
    choose_shape(C, block_threads, &kc, sh.cb_max);
    kc.minb = min_blocks ? min_blocks : default_min_blocks(kc, lop3);
    kc.sync_every = sync_of(sh);
    pl->d = d; pl->C = C; pl->bp = bp; pl->ep = ep;
    return NSAT_OK;
}

struct QsatPlan {
    KernelConfig kc;
    std::vector<uint8_t> q;   // padded quantifiers
    uint32_t n = 0, d = 0, np = 0, C = 0, A = 0;
    uint32_t s = 0;           // fixed prefix bits (inputs 0..s-1)
    uint32_t fsub = 0;        // first quantifier block of the problem below the prefix
    uint32_t m = 0;           // unit level: np - (s + fsub)
};

int plan_qsat(uint32_t n, const std::vector<uint8_t>& quants_in, bool data, uint32_t chunk_bits,
              const Shape& sh, uint32_t prefix_bits, QsatPlan* pl, std::string* err, uint32_t lop3 = 0) {
    const uint32_t block_threads = sh.block_threads, min_blocks = sh.min_blocks;
    if (quants_in.size() != n || n == 0) { *err = "quantifier count differs from inputs"; return NSAT_EINVAL; }
    if (prefix_bits >= n) { *err = "prefix must leave at least one free input"; return NSAT_EINVAL; }
    // dummy innermost inputs (the opposite quantifier of the last one: no
    // effect on value or witness) for circuits of fewer than 15 inputs, and
    // for sub-problems that leave fewer than 10 inputs below the prefix
    const uint32_t d = std::max<uint32_t>(n < 15 ? 15 - n : 0, n - prefix_bits < 10 ? 10 - (n - prefix_bits) : 0);
    const uint32_t np = n + d;
    if (np > 128) { *err = "too many inputs"; return NSAT_EUNSUPPORTED; }
    std::vector<uint8_t> q = quants_in;
    for (uint32_t k = 0; k < d; k++) q.push_back(quants_in[n - 1] ? 0 : 1);
    const uint32_t s = prefix_bits;
    uint32_t fsub = 0;
    while (s + fsub < n && q[s + fsub] == q[s]) fsub++;
    if (fsub > 64) { *err = "first quantifier block longer than 64"; return NSAT_EUNSUPPORTED; }
    const uint32_t m = np - (s + fsub);
    uint32_t C = chunk_bits ? std::max<uint32_t>(15, chunk_bits + d) : 34;
    C = std::min<uint32_t>(C, np - s);
    if (C < 10) { *err = "prefix leaves fewer than 2^10 assignments"; return NSAT_EINVAL; }
    const uint32_t A = np - C;
    if (A - s > 64) { *err = "more than 64 quantifiers above one launch"; return NSAT_EUNSUPPORTED; }
    KernelConfig& kc = pl->kc;
    kc.mode = Mode::QSAT;
    kc.data = data;
    kc.nin = np;
    kc.nb = np;
    kc.in_of_bit.resize(np);
    for (uint32_t p = 0; p < np; p++) {
        int in = (int)(np - 1 - p);
        kc.in_of_bit[p] = (data || in >= (int)n) ? -1 : in;
    }
    choose_shape(C, block_threads, &kc, sh.cb_max);
    kc.minb = min_blocks ? min_blocks : default_min_blocks(kc, lop3);
    kc.sync_every = sync_of(sh);
    kc.m = std::min<uint32_t>(m, 127);
    kc.q0all = q[s] != 0;
    kc.allbits = 0;
    for (uint32_t j = 0; j < std::min<uint32_t>(C, 64); j++)
        if (q[np - 1 - j]) kc.allbits |= 1ull << j;
    pl->q = q; pl->n = n; pl->d = d; pl->np = np; pl->C = C; pl->A = A;
    pl->s = s; pl->fsub = fsub; pl->m = m;
    return NSAT_OK;
}

// chunked: the partitioned solver builds u64 entries chunk by chunk, so the
// device-memory limit on n does not apply.
int plan_table(const Circuit& circ, bool steps, KernelConfig* kc, std::string* err, bool chunked = false) {
    const uint32_t n = circ.n;
    if (circ.outputs.size() != n + 1) { *err = "SATOSTOP circuit needs n+1 outputs"; return NSAT_EINVAL; }
    if (!chunked && n > 36) { *err = "state longer than 36 bits does not fit device memory"; return NSAT_EUNSUPPORTED; }
    if (n > 62) { *err = "state longer than 62 bits"; return NSAT_EUNSUPPORTED; }
    uint32_t fmt;
    if (steps) {
        if (n > 31) { *err = "steps need n <= 31"; return NSAT_EUNSUPPORTED; }
        fmt = 2;
    } else {
        fmt = (n <= 31 && !chunked) ? 0 : 1;
    }
    kc->mode = Mode::TABLE;
    kc->nin = n;
    kc->nb = n;
    kc->in_of_bit.resize(n);
    for (uint32_t p = 0; p < n; p++) kc->in_of_bit[p] = (int)p;
    kc->wb = 3;
    kc->fmt = fmt;
    kc->nout = n + 1;
    return NSAT_OK;
}

}  // namespace

// ---------------------------------------------------------------------------
// context

extern "C" int nsat_device_count(void) {
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) { cudaGetLastError(); return 0; }
    return n;
}

extern "C" const char* nsat_strerror(int s) {
    switch (s) {
    case NSAT_OK: return "ok";
    case NSAT_EINVAL: return "invalid argument";
    case NSAT_ENOMEM: return "out of memory";
    case NSAT_ECOMPILE: return "kernel compile failed";
    case NSAT_ECUDA: return "CUDA error";
    case NSAT_ETIMEOUT: return "device wait timed out";
    case NSAT_ENODEV: return "no CUDA device";
    case NSAT_EUNSUPPORTED: return "unsupported size";
    case NSAT_EPARSE: return "parse error";
    case NSAT_EBUSY: return "busy";
    default: return "unknown status";
    }
}

extern "C" const char* nsat_last_error(const nsat_ctx* ctx) { return ctx ? ctx->last_err.c_str() : ""; }

extern "C" int nsat_create(int device, const nsat_opts* opts, nsat_ctx** out) {
    if (!out) return NSAT_EINVAL;
    *out = nullptr;
    int ndev = nsat_device_count();
    if (ndev <= 0) return NSAT_ENODEV;
    if (device < 0 || device >= ndev) return NSAT_EINVAL;
    std::unique_ptr<nsat_ctx> c(new nsat_ctx());
    nsat_ctx* ctx = c.get();
    ctx->device = device;
    if (opts) ctx->opts = *opts;
    if (set_device(ctx)) return NSAT_ECUDA;
    CK(cudaFree(nullptr));
    CK(cudaDeviceGetAttribute(&ctx->sm_count, cudaDevAttrMultiProcessorCount, device));
    CK(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
    cudaMemPoolProps pp{};
    pp.allocType = cudaMemAllocationTypePinned;
    pp.handleTypes = cudaMemHandleTypeNone;
    pp.location.type = cudaMemLocationTypeDevice;
    pp.location.id = device;
    CK(cudaMemPoolCreate(&ctx->pool, &pp));
    uint64_t keep = kPoolKeepBytes;
    CK(cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &keep));
    CK(cudaMalloc(&ctx->d_out, sizeof(LaunchOut) * kRing));
    CK(cudaMallocHost(&ctx->h_out, sizeof(LaunchOut) * kRing));
    CK(cudaMallocHost(&ctx->h_init, sizeof(LaunchOut)));
    CK(cudaMalloc(&ctx->d_join, sizeof(NsatJoinState)));
    CK(cudaMallocHost(&ctx->h_join, sizeof(NsatJoinState)));
    memset(ctx->h_init, 0, sizeof(LaunchOut));
    ctx->h_init->min_idx = ~0ull;
    for (int i = 0; i < kRing; i++) {
        CK(cudaEventCreate(&ctx->ev0[i]));
        CK(cudaEventCreate(&ctx->ev1[i]));
        CK(cudaEventCreateWithFlags(&ctx->evd[i], cudaEventDisableTiming));
    }
    std::string err;
    if (!driver_api(&err)) return NSAT_ECUDA;
    *out = c.release();
    return NSAT_OK;
}

extern "C" void nsat_destroy(nsat_ctx* ctx) {
    if (!ctx) return;
    cudaSetDevice(ctx->device);
    if (ctx->stream) cudaStreamSynchronize(ctx->stream);
    for (int i = 0; i < kRing; i++) {
        if (ctx->ev0[i]) cudaEventDestroy(ctx->ev0[i]);
        if (ctx->ev1[i]) cudaEventDestroy(ctx->ev1[i]);
        if (ctx->evd[i]) cudaEventDestroy(ctx->evd[i]);
    }
    cudaFree(ctx->d_out);
    cudaFreeHost(ctx->h_out);
    cudaFreeHost(ctx->h_init);
    cudaFree(ctx->d_scratch);
    cudaFree(ctx->d_data);
    cudaFree(ctx->d_join);
    cudaFreeHost(ctx->h_join);
    if (ctx->stream) cudaStreamDestroy(ctx->stream);
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
}

// ---------------------------------------------------------------------------
// circuits and text

extern "C" int nsat_circuit_new(nsat_ctx* ctx, const nsat_circuit_desc* desc, nsat_circuit** out) {
    if (!ctx || !desc || !out || (desc->gate_num && !desc->gates) || !desc->outputs) return NSAT_EINVAL;
    *out = nullptr;
    for (uint32_t k = 0; k < desc->gate_num; k++)
        if (desc->gates[3 * k] > 3) return fail(ctx, NSAT_EINVAL, "bad gate function");
    Circuit c = from_desc(desc);
    std::string v = c.validate();
    if (!v.empty()) return fail(ctx, NSAT_EINVAL, v);
    nsat_circuit* nc = new nsat_circuit();
    nc->ctx = ctx;
    nc->device = ctx->device;
    nc->circ = std::move(c);
    *out = nc;
    return NSAT_OK;
}

extern "C" void nsat_circuit_free(nsat_circuit* c) {
    if (!c) return;
    // The handle may hold the last reference to its kernels' modules: release
    // them with their device current (solves return only after their launches
    // finished, so none is queued), then give the caller back its device.
    int prev = -1;
    const bool switched = cudaGetDevice(&prev) == cudaSuccess && c->device >= 0 && c->device != prev &&
                          cudaSetDevice(c->device) == cudaSuccess;
    delete c;
    if (switched) cudaSetDevice(prev);
}

extern "C" int nsat_circuit_stats(nsat_ctx* ctx, nsat_circuit* c, int output, uint32_t* live,
                                  uint32_t* ops) {
    if (!ctx || !c) return NSAT_EINVAL;
    std::vector<uint32_t> which;
    if (output < 0) for (uint32_t j = 0; j < c->circ.outputs.size(); j++) which.push_back(j);
    else if ((size_t)output < c->circ.outputs.size()) which.push_back((uint32_t)output);
    else return NSAT_EINVAL;
    const LutNet& net = get_net(c, which);
    if (live) *live = net.live_gates;
    if (ops) *ops = (uint32_t)net.luts.size();
    return NSAT_OK;
}

extern "C" int nsat_parse(const char* text, size_t len, nsat_parsed** out) {
    if (!text || !out) return NSAT_EINVAL;
    *out = nullptr;
    std::unique_ptr<nsat_parsed> p(new nsat_parsed());
    std::string err;
    if (!parse_gatesim(std::string(text, len), &p->p, &err)) return NSAT_EPARSE;
    for (const Gate& g : p->p.circuit.gates) { p->gates.push_back(g.func); p->gates.push_back(g.i0); p->gates.push_back(g.i1); }
    for (const Output& o : p->p.circuit.outputs) { p->outputs.push_back(o.wire); p->outputs.push_back(o.neg); }
    *out = p.release();
    return NSAT_OK;
}

extern "C" int nsat_parsed_get(const nsat_parsed* p, nsat_circuit_desc* d, const uint8_t** quants) {
    if (!p || !d) return NSAT_EINVAL;
    d->input_len = p->p.circuit.n;
    d->gate_num = (uint32_t)p->p.circuit.gates.size();
    d->gates = p->gates.data();
    d->output_num = (uint32_t)p->p.circuit.outputs.size();
    d->outputs = p->outputs.data();
    if (quants) *quants = p->p.quants.empty() ? nullptr : p->p.quants.data();
    return NSAT_OK;
}

extern "C" void nsat_parsed_free(nsat_parsed* p) { delete p; }

extern "C" int nsat_format(const nsat_circuit_desc* desc, const uint8_t* quants, char* buf, size_t buflen,
                           size_t* needed) {
    if (!desc) return NSAT_EINVAL;
    Circuit c = from_desc(desc);
    if (!c.validate().empty()) return NSAT_EINVAL;
    std::vector<uint8_t> q;
    if (quants) q.assign(quants, quants + c.n);
    std::string s = format_gatesim(c, quants ? &q : nullptr);
    if (needed) *needed = s.size();
    if (buf && buflen) {
        size_t k = std::min(buflen - 1, s.size());
        memcpy(buf, s.data(), k);
        buf[k] = 0;
        if (k < s.size()) return NSAT_EINVAL;
    }
    return NSAT_OK;
}

// ---------------------------------------------------------------------------
// SAT

extern "C" int nsat_sat_solve(nsat_ctx* ctx, nsat_circuit* c, const nsat_sat_opts* opts,
                              nsat_sat_result* res) {
    if (!ctx || !c || !res) return NSAT_EINVAL;
    memset(res, 0, sizeof(*res));
    const double t_start = now_ms();
    if (int rc = set_device(ctx)) return rc;
    nsat_sat_opts o{};
    if (opts) o = *opts;
    SatPlan plan;
    std::string perr;
    const std::vector<uint32_t> out0{0};
    const LutNet& net = get_net(c, out0);
    if (int rc = plan_sat(c->circ.n, o, effective_shape(ctx, c->tuned), &plan, &perr, (uint32_t)net.luts.size()))
        return fail(ctx, rc, perr);
    const KernelConfig& kc = plan.kc;
    const uint32_t d = plan.d, C = plan.C;
    const u128 bp = plan.bp, ep = plan.ep;
    CUfunction fn;
    std::shared_ptr<JitModule> mod;
    if (int rc = get_circuit_kernel(ctx, c, out0, kc, net, "nsat_sat", &fn, &mod)) return rc;
    const uint64_t L0 = (uint64_t)(bp >> C);
    const uint64_t nl = (uint64_t)((ep - bp) >> C);
    const unsigned grid = 1u << kc.cb, threads = kc.threads();
    u128 count = 0;
    bool found = false;
    u128 witness = 0;
    uint64_t consumed = 0;
    double dev_ms = 0;
    uint32_t launches = 0;
    uint64_t launch_idx_buf[kRing];
    uint64_t chunk_of_slot[kRing];
    LaunchOut* d_out = ctx->d_out;
    nsat_sat_share* share = o.find_all ? nullptr : o.share;
    int rc = run_ring(
        ctx, nl,
        [&](uint64_t k, int slot) {
            launch_idx_buf[slot] = L0 + (share ? chunk_of_slot[slot] : k);
            LaunchOut* po = d_out + slot;
            void* params[] = {&launch_idx_buf[slot], &po};
            return launch(ctx, fn, grid, threads, params);
        },
        [&](uint64_t k, const LaunchOut& r) {
            const uint64_t chunk = share ? chunk_of_slot[k % kRing] : k;
            consumed++;
            count += r.count;
            if (r.min_idx != ~0ull) {
                const u128 w = (((u128)(L0 + chunk)) << C) + r.min_idx;
                if (!found || w < witness) witness = w;
                found = true;
                if (share) {
                    // no participant claims this chunk or a later one any more
                    uint64_t cur = __atomic_load_n(&share->stop_plus1, __ATOMIC_ACQUIRE);
                    while ((cur == 0 || chunk + 1 < cur) &&
                           !__atomic_compare_exchange_n(&share->stop_plus1, &cur, chunk + 1, false, __ATOMIC_ACQ_REL,
                                                        __ATOMIC_ACQUIRE)) {
                    }
                }
            }
            // with a shared queue every issued chunk is consumed: a lower
            // one in flight may hold a lower witness
            return share ? true : !(found && !o.find_all);
        },
        &dev_ms, &launches,
        [&](uint64_t, int slot) {
            if (!share) return true;
            const uint64_t c = __atomic_fetch_add(&share->next, 1, __ATOMIC_ACQ_REL);
            const uint64_t st = __atomic_load_n(&share->stop_plus1, __ATOMIC_ACQUIRE);
            if (c >= nl || (st != 0 && c + 1 >= st)) return false;
            chunk_of_slot[slot] = c;
            return true;
        });
    if (rc) return rc;
    res->satisfiable = found ? 1 : 0;
    const u128 cnt = count >> d;
    res->count_lo = (uint64_t)cnt;
    res->count_hi = (uint64_t)(cnt >> 64);
    const u128 w = witness >> d;
    res->witness_lo = found ? (uint64_t)w : 0;
    res->witness_hi = found ? (uint64_t)(w >> 64) : 0;
    const u128 sc = ((u128)consumed << C) >> d;
    res->scanned_lo = (uint64_t)sc;
    res->scanned_hi = (uint64_t)(sc >> 64);
    res->device_ms = dev_ms;
    res->launches = launches;
    res->wall_ms = now_ms() - t_start;
    return NSAT_OK;
}

// ---------------------------------------------------------------------------
// QSAT

namespace {

// With prefix_count > 1 (one launch per prefix only), solves the sub-problems
// under prefixes prefix .. prefix + prefix_count - 1 back to back through the
// launch ring and hands each one's result, in order, to on_block, which
// returns false to stop; res then holds the last one handed over.
int qsat_common(nsat_ctx* ctx, nsat_circuit* c, const std::vector<uint8_t>& quants_in,
                const uint32_t* data_words, uint32_t n_items_bits, uint32_t chunk_bits,
                nsat_qsat_result* res, unsigned char* fixed_scratch = nullptr,
                size_t fixed_scratch_bytes = 0, uint32_t prefix_bits = 0, uint64_t prefix = 0,
                uint64_t prefix_count = 1,
                const std::function<bool(uint64_t, const nsat_qsat_result&)>* on_block = nullptr) {
    memset(res, 0, sizeof(*res));
    const double t_start = now_ms();
    if (int rc = set_device(ctx)) return rc;
    const bool data = data_words != nullptr;
    const uint32_t n = data ? n_items_bits : c->circ.n;
    QsatPlan plan;
    std::string perr;
    LutNet empty;
    const std::vector<uint32_t> out0{0};
    const LutNet& net = data ? empty : get_net(c, out0);
    const Shape sh = data ? effective_shape(ctx, Shape()) : effective_shape(ctx, c->tuned_qsat);
    if (int rc = plan_qsat(n, quants_in, data, chunk_bits, sh, prefix_bits, &plan, &perr,
                           data ? 0u : (uint32_t)net.luts.size()))
        return fail(ctx, rc, perr);
    if (prefix_bits < 64 && (prefix >> prefix_bits) != 0) return fail(ctx, NSAT_EINVAL, "prefix wider than prefix_bits");
    const KernelConfig& kc = plan.kc;
    // a launch the fixed area cannot hold is refused before any kernel is compiled or loaded
    if (fixed_scratch && ((size_t)2 << kc.cb) > fixed_scratch_bytes)
        return fail(ctx, NSAT_EUNSUPPORTED,
                    "launch needs " + std::to_string((size_t)2 << kc.cb) + " scratch bytes, the fixed area holds " +
                    std::to_string(fixed_scratch_bytes) + " (use smaller chunk_bits)");
    const std::vector<uint8_t>& q = plan.q;
    // below a fixed prefix of s inputs the problem is the sub-formula over
    // inputs s..n-1: its first block has fsub inputs and As quantifiers lie
    // above one launch
    const uint32_t d = plan.d, np = plan.np, m = plan.m, C = plan.C, s = plan.s, f = plan.fsub;
    const uint32_t A = plan.A - s;
    const uint64_t L0 = s ? (prefix << A) : 0;
    CUfunction fn;
    std::shared_ptr<JitModule> mod;
    if (int rc = data ? get_kernel(ctx, kc, net, "nsat_qsat", &fn, &mod)
                      : get_circuit_kernel(ctx, c, out0, kc, net, "nsat_qsat", &fn, &mod))
        return rc;
    if (!fixed_scratch) {
        if (int rc = ensure_scratch(ctx, (size_t)2 << kc.cb)) return rc;
    }
    if (data) {
        // expand 2^n items to 2^np (each item repeated 2^d times)
        const uint64_t nw = 1ull << (np - 5);
        std::vector<uint32_t> ex(nw, 0);
        for (uint64_t v = 0; v < (1ull << np); v++) {
            uint64_t src = v >> d;
            if ((data_words[src >> 5] >> (src & 31)) & 1u) ex[v >> 5] |= 1u << (v & 31);
        }
        if (ctx->data_bytes < nw * 4) {
            cudaFree(ctx->d_data);
            ctx->d_data = nullptr;
            ctx->data_bytes = 0;
            CK(cudaMalloc(&ctx->d_data, nw * 4));
            ctx->data_bytes = nw * 4;
        }
        CK(cudaMemcpyAsync(ctx->d_data, ex.data(), nw * 4, cudaMemcpyHostToDevice, ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
    }
    if (prefix_count > 1 && (A != 0 || !on_block || (prefix_bits < 64 && prefix + prefix_count > (1ull << prefix_bits))))
        return fail(ctx, NSAT_EUNSUPPORTED, "a run of prefixes needs one launch per prefix");
    const bool q0all = q[s] != 0;
    const bool dec = !q0all;   // value of a decisive unit
    std::unique_ptr<QuantReducer> qr;
    if (A > 0) qr.reset(new QuantReducer(std::vector<uint8_t>(q.begin() + s, q.begin() + s + A)));
    FinalResult fr;
    bool have = false;
    uint64_t nl = prefix_count > 1 ? prefix_count : (A == 64 ? ~0ull : (1ull << A));
    const unsigned grid = 1u << kc.cb, threads = kc.threads();
    uint64_t launch_idx_buf[kRing];
    LaunchOut* d_out = ctx->d_out;
    unsigned char* scratch = fixed_scratch ? fixed_scratch : ctx->d_scratch;
    const uint32_t* dd = ctx->d_data;
    double dev_ms = 0;
    uint32_t launches = 0;
    int rc = run_ring(
        ctx, nl,
        [&](uint64_t k, int slot) {
            launch_idx_buf[slot] = L0 + k;
            LaunchOut* po = d_out + slot;
            void* params[] = {&launch_idx_buf[slot], &po, &scratch, &dd};
            return launch(ctx, fn, grid, threads, params);
        },
        [&](uint64_t k, const LaunchOut& r) {
            if (A == 0) {
                fr.reversed = q0all;
                fr.solution_bits = f;
                fr.has_solution = r.min_idx != ~0ull;
                fr.solution = fr.has_solution ? reverse_bits(r.min_idx, f) : 0;
                have = true;
                if (prefix_count > 1) {
                    nsat_qsat_result b{};
                    b.reversed = fr.reversed;
                    b.solution_bits = fr.solution_bits;
                    b.has_solution = fr.has_solution;
                    b.value = fr.has_solution ? (q0all ? 0 : 1) : (q0all ? 1 : 0);
                    b.solution_lo = fr.solution;
                    return (*on_block)(prefix + k, b);
                }
                return false;
            }
            bool value;
            if (m < C) value = (r.min_idx != ~0ull) ? dec : !dec;
            else value = r.tree != 0;
            qr->push(value);
            FinalResult t;
            if (qr->final_result(&t)) {
                fr.reversed = q0all;
                fr.solution_bits = f;
                fr.has_solution = t.has_solution;
                if (t.has_solution && f > A)
                    fr.solution = t.solution | (reverse_bits(r.min_idx, f - A) << A);
                else
                    fr.solution = t.has_solution ? t.solution : 0;
                have = true;
                (void)k;
                return false;
            }
            return true;
        },
        &dev_ms, &launches);
    if (rc) return rc;
    if (!have) return fail(ctx, NSAT_ECUDA, "QSAT reduction did not finish");
    res->reversed = fr.reversed;
    res->solution_bits = fr.solution_bits;
    res->has_solution = fr.has_solution;
    res->value = fr.has_solution ? (q0all ? 0 : 1) : (q0all ? 1 : 0);
    res->solution_lo = fr.solution;
    res->solution_hi = 0;
    res->launches = launches;
    res->chunk_bits = C - d;
    res->scanned = (uint64_t)(((u128)launches << C) >> d);
    res->device_ms = dev_ms;
    res->wall_ms = now_ms() - t_start;
    return NSAT_OK;
}

}  // namespace

extern "C" int nsat_qsat_solve(nsat_ctx* ctx, nsat_circuit* c, const uint8_t* quants,
                               const nsat_qsat_opts* opts, nsat_qsat_result* res) {
    if (!ctx || !c || !quants || !res) return NSAT_EINVAL;
    std::vector<uint8_t> q(quants, quants + c->circ.n);
    for (auto& v : q) v = v ? 1 : 0;
    uint32_t f = 0;
    while (f < q.size() && q[f] == q[0]) f++;
    if (f > 64) return fail(ctx, NSAT_EUNSUPPORTED, "first quantifier block longer than 64");
    return qsat_common(ctx, c, q, nullptr, 0, opts ? opts->chunk_bits : 0, res, nullptr, 0,
                       opts ? opts->prefix_bits : 0, opts ? opts->prefix : 0);
}

int nsat::qsat_solve_blocks(nsat_ctx* ctx, nsat_circuit* c, const uint8_t* quants, uint32_t prefix_bits,
                            uint64_t first, uint64_t count,
                            const std::function<bool(uint64_t, const nsat_qsat_result&)>& on_block) {
    if (!ctx || !c || !quants || count == 0) return NSAT_EINVAL;
    std::vector<uint8_t> q(quants, quants + c->circ.n);
    for (auto& v : q) v = v ? 1 : 0;
    nsat_qsat_result last{};
    if (count == 1) {
        int rc = qsat_common(ctx, c, q, nullptr, 0, 0, &last, nullptr, 0, prefix_bits, first);
        if (rc == NSAT_OK) on_block(first, last);
        return rc;
    }
    return qsat_common(ctx, c, q, nullptr, 0, 0, &last, nullptr, 0, prefix_bits, first, count, &on_block);
}

int nsat::ctx_device(const nsat_ctx* ctx) { return ctx ? ctx->device : -1; }
cudaStream_t nsat::ctx_stream(const nsat_ctx* ctx) { return ctx->stream; }
cudaError_t nsat::ctx_alloc(nsat_ctx* ctx, void** p, size_t bytes) {
    return cudaMallocFromPoolAsync(p, bytes, ctx->pool, ctx->stream);
}
void nsat::ctx_free(nsat_ctx* ctx, void* p) {
    if (p) cudaFreeAsync(p, ctx->stream);
}
void nsat::ctx_trim(nsat_ctx* ctx) {
    cudaStreamSynchronize(ctx->stream);
    cudaMemPoolTrimTo(ctx->pool, 0);
}
int nsat::ctx_sm_count(const nsat_ctx* ctx) { return ctx->sm_count; }
bool nsat::ctx_no_optimize(const nsat_ctx* ctx) { return ctx->opts.no_optimize != 0; }
nsat_opts nsat::ctx_opts(const nsat_ctx* ctx) { return ctx->opts; }
int nsat::ctx_fail(nsat_ctx* ctx, int code, const std::string& msg) { return fail(ctx, code, msg); }
Circuit nsat::circuit_from_desc(const nsat_circuit_desc* d) { return from_desc(d); }

int nsat::qsat_solve_with_scratch(nsat_ctx* ctx, nsat_circuit* c, const uint8_t* quants,
                                   const nsat_qsat_opts* opts, nsat_qsat_result* res,
                                   unsigned char* scratch, size_t scratch_bytes) {
    if (!ctx || !c || !quants || !res || !scratch) return NSAT_EINVAL;
    std::vector<uint8_t> q(quants, quants + c->circ.n);
    for (auto& v : q) v = v ? 1 : 0;
    uint32_t f = 0;
    while (f < q.size() && q[f] == q[0]) f++;
    if (f > 64) return fail(ctx, NSAT_EUNSUPPORTED, "first quantifier block longer than 64");
    return qsat_common(ctx, c, q, nullptr, 0, opts ? opts->chunk_bits : 0, res, scratch, scratch_bytes,
                       opts ? opts->prefix_bits : 0, opts ? opts->prefix : 0);
}

extern "C" int nsat_qsat_reduce_words(nsat_ctx* ctx, const uint8_t* quants, uint32_t nq,
                                      const uint32_t* words, nsat_qsat_result* res) {
    if (!ctx || !quants || !words || !res || nq < 5 || nq > 30) return NSAT_EINVAL;
    std::vector<uint8_t> q(quants, quants + nq);
    for (auto& v : q) v = v ? 1 : 0;
    return qsat_common(ctx, nullptr, q, words, nq, 0, res);
}

// ---------------------------------------------------------------------------
// SATOSTOP

extern "C" int nsat_stop_table_build(nsat_ctx* ctx, nsat_circuit* c, const nsat_table_opts* opts,
                                     nsat_table** out) {
    if (!ctx || !c || !out) return NSAT_EINVAL;
    *out = nullptr;
    if (int rc = set_device(ctx)) return rc;
    const uint32_t n = c->circ.n;
    KernelConfig kc;
    std::string perr;
    if (int rc = plan_table(c->circ, opts && opts->want_steps, &kc, &perr)) return fail(ctx, rc, perr);
    std::unique_ptr<nsat_table> t(new nsat_table());
    t->ctx = ctx;
    t->n = n;
    t->fmt = kc.fmt;
    t->N = 1ull << n;
    t->entry_bytes = kc.fmt == 0 ? 4 : 8;
    const size_t bytes = std::max<size_t>(t->N * t->entry_bytes, 256);
    for (int i = 0; i < 2; i++) {
        cudaError_t e = ctx_alloc(ctx, &t->buf[i], bytes);
        if (e != cudaSuccess) {
            t->buf[i] = nullptr;
            cudaGetLastError();
            return fail(ctx, NSAT_ENOMEM, "table allocation failed");
        }
    }
    std::vector<uint32_t> which;
    for (uint32_t j = 0; j <= n; j++) which.push_back(j);
    const LutNet& net = get_net(c, which);
    CUfunction fn;
    std::shared_ptr<JitModule> mod;
    if (int rc = get_circuit_kernel(ctx, c, which, kc, net, "nsat_table", &fn, &mod)) return rc;
    uint64_t nwords = n >= 5 ? (t->N >> 5) : 1;
    const unsigned threads = kc.threads();
    uint64_t want = (nwords + threads - 1) / threads;
    unsigned grid = (unsigned)std::min<uint64_t>(want, (uint64_t)ctx->sm_count * 16);
    LaunchOut* po = ctx->d_out;
    void* tb = t->buf[0];
    uint64_t w0 = 0;
    void* params[] = {&nwords, &w0, &tb, &po};
    CK(cudaMemcpyAsync(ctx->d_out, ctx->h_init, sizeof(LaunchOut), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaEventRecord(ctx->ev0[0], ctx->stream));
    if (int rc = launch(ctx, fn, grid, threads, params)) return rc;
    CK(cudaEventRecord(ctx->ev1[0], ctx->stream));
    CK(cudaMemcpyAsync(ctx->h_out, ctx->d_out, sizeof(LaunchOut), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ctx->ev0[0], ctx->ev1[0]));
    t->build_ms = ms;
    t->any_stop = ctx->h_out[0].any != 0;
    t->cur = 0;
    *out = t.release();
    return NSAT_OK;
}

namespace nsat {

int table_chunk_u64(nsat_ctx* ctx, nsat_circuit* c, uint64_t first_state, uint64_t count, uint64_t* dev_out,
                    uint32_t* any_stop, float* ms) {
    if (int rc = set_device(ctx)) return rc;
    KernelConfig kc;
    std::string perr;
    if (int rc = plan_table(c->circ, false, &kc, &perr, true)) return fail(ctx, rc, perr);
    const uint32_t n = c->circ.n;
    if (n < 5 || (first_state & 31) || (count & 31) || count == 0)
        return fail(ctx, NSAT_EINVAL, "table chunks are whole 32-state words");
    std::vector<uint32_t> which;
    for (uint32_t j = 0; j <= n; j++) which.push_back(j);
    const LutNet& net = get_net(c, which);
    CUfunction fn;
    std::shared_ptr<JitModule> mod;
    if (int rc = get_circuit_kernel(ctx, c, which, kc, net, "nsat_table", &fn, &mod)) return rc;
    uint64_t nwords = count >> 5, w0 = first_state >> 5;
    const unsigned threads = kc.threads();
    const uint64_t want = (nwords + threads - 1) / threads;
    const unsigned grid = (unsigned)std::min<uint64_t>(want, (uint64_t)ctx->sm_count * 16);
    LaunchOut* po = ctx->d_out;
    void* tb = dev_out;
    void* params[] = {&nwords, &w0, &tb, &po};
    CK(cudaMemcpyAsync(ctx->d_out, ctx->h_init, sizeof(LaunchOut), cudaMemcpyHostToDevice, ctx->stream));
    CK(cudaEventRecord(ctx->ev0[0], ctx->stream));
    if (int rc = launch(ctx, fn, grid, threads, params)) return rc;
    CK(cudaEventRecord(ctx->ev1[0], ctx->stream));
    CK(cudaMemcpyAsync(ctx->h_out, ctx->d_out, sizeof(LaunchOut), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    if (ms) CK(cudaEventElapsedTime(ms, ctx->ev0[0], ctx->ev1[0]));
    if (any_stop) *any_stop = ctx->h_out[0].any != 0;
    return NSAT_OK;
}

const Circuit& circuit_of(const nsat_circuit* c) { return c->circ; }

}  // namespace nsat

extern "C" void nsat_table_free(nsat_table* t) { delete t; }

extern "C" uint64_t nsat_table_bytes(const nsat_table* t) {
    return t ? 2ull * std::max<uint64_t>(t->N * t->entry_bytes, 256) : 0;
}

extern "C" int nsat_table_read(nsat_table* t, uint64_t first, uint64_t count, uint64_t* out) {
    if (!t || !out || first > t->N || count > t->N - first) return NSAT_EINVAL;
    nsat_ctx* ctx = t->ctx;
    if (int rc = set_device(ctx)) return rc;
    const uint64_t mask = (t->fmt == 2) ? 0xffffffffull : ~0ull;
    if (t->entry_bytes == 4) {
        std::vector<uint32_t> tmp(count);
        CK(cudaMemcpy(tmp.data(), (uint32_t*)t->buf[t->cur] + first, count * 4, cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < count; i++) out[i] = tmp[i];
    } else {
        CK(cudaMemcpy(out, (uint64_t*)t->buf[t->cur] + first, count * 8, cudaMemcpyDeviceToHost));
        for (uint64_t i = 0; i < count; i++) out[i] &= mask;
    }
    return NSAT_OK;
}

extern "C" int nsat_stop_solve(nsat_ctx* ctx, nsat_table* t, const nsat_stop_opts* opts,
                               nsat_stop_result* res) {
    if (!ctx || !t || !opts || !res || t->ctx != ctx) return NSAT_EINVAL;
    memset(res, 0, sizeof(*res));
    if (opts->unknowns > t->n || opts->mode > 1) return NSAT_EINVAL;
    if (int rc = set_device(ctx)) return rc;
    res->build_ms = t->build_ms;
    if (!t->any_stop) return NSAT_OK;   // check_stop: no state ever stops
    NsatJoinState* h = ctx->h_join;
    memset(h, 0, sizeof(*h));
    for (int i = 0; i < 72; i++) h->best[i] = ~0ull;
    CK(cudaMemcpyAsync(ctx->d_join, h, sizeof(*h), cudaMemcpyHostToDevice, ctx->stream));
    const uint32_t n = t->n;
    CK(cudaEventRecord(ctx->ev0[0], ctx->stream));
    int src = t->cur;
    for (uint32_t r = 1; r <= n; r++) {
        int rc = nsat_launch_join_round((int)t->fmt, t->buf[src], t->buf[src ^ 1], t->N, n, opts->unknowns, r,
                                        opts->mode, ctx->d_join, ctx->sm_count, ctx->stream);
        if (rc) return fail(ctx, NSAT_ECUDA, "join launch failed");
        src ^= 1;
    }
    CK(cudaEventRecord(ctx->ev1[0], ctx->stream));
    CK(cudaMemcpyAsync(h, ctx->d_join, sizeof(*h), cudaMemcpyDeviceToHost, ctx->stream));
    CK(cudaStreamSynchronize(ctx->stream));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, ctx->ev0[0], ctx->ev1[0]));
    res->join_ms = ms;
    const uint32_t fr = h->final_round ? h->final_round : n;
    const uint64_t best = h->best[fr];
    res->rounds = fr;
    // round r wrote buffer cur0 ^ (r & 1); rounds after an early exit write nothing
    const int buf = t->cur ^ (int)(fr & 1);
    t->cur = buf;
    if (best != ~0ull) {
        uint64_t e = 0;
        if (t->entry_bytes == 4) {
            uint32_t v;
            CK(cudaMemcpy(&v, (uint32_t*)t->buf[buf] + best, 4, cudaMemcpyDeviceToHost));
            e = v;
        } else {
            CK(cudaMemcpy(&e, (uint64_t*)t->buf[buf] + best, 8, cudaMemcpyDeviceToHost));
        }
        res->found = 1;
        res->start = best;
        res->end = e & ((1ull << n) - 1);
        res->steps = t->fmt == 2 ? (e >> 32) : 0;
    }
    return NSAT_OK;
}

// ---------------------------------------------------------------------------
// measurement

extern "C" int nsat_probe_lop3_peak(nsat_ctx* ctx, double* lop3_per_s, double* sm_mhz) {
    if (!ctx || !lop3_per_s) return NSAT_EINVAL;
    if (int rc = set_device(ctx)) return rc;
    const int blocks = ctx->sm_count * 8, iters = 1 << 14;
    uint32_t* dbuf = nullptr;
    uint64_t* dclk = nullptr;
    CK(cudaMalloc(&dbuf, (size_t)blocks * 256 * 4));
    CK(cudaMalloc(&dclk, 24 * (size_t)blocks));
    std::vector<uint64_t> hclk(3 * (size_t)blocks);
    double best = 0, mhz = 0;
    for (int rep = 0; rep < 3; rep++) {
        CK(cudaEventRecord(ctx->ev0[0], ctx->stream));
        if (nsat_launch_lop3_probe(dbuf, blocks, iters, dclk, ctx->stream)) {
            cudaFree(dbuf); cudaFree(dclk);
            return fail(ctx, NSAT_ECUDA, "probe launch failed");
        }
        CK(cudaEventRecord(ctx->ev1[0], ctx->stream));
        CK(cudaStreamSynchronize(ctx->stream));
        float ms = 0;
        CK(cudaEventElapsedTime(&ms, ctx->ev0[0], ctx->ev1[0]));
        CK(cudaMemcpy(hclk.data(), dclk, 24 * (size_t)blocks, cudaMemcpyDeviceToHost));
        // per SM: cycles from the first block's loop start to the last
        // block's loop end (clock64 is a per-SM counter), averaged over SMs
        std::map<uint64_t, std::pair<uint64_t, uint64_t>> span;
        for (int b = 0; b < blocks; b++) {
            const uint64_t c0 = hclk[3 * b], c1 = hclk[3 * b + 1], sm = hclk[3 * b + 2];
            auto it = span.find(sm);
            if (it == span.end()) span[sm] = {c0, c1};
            else { it->second.first = std::min(it->second.first, c0); it->second.second = std::max(it->second.second, c1); }
        }
        double cyc = 0;
        for (auto& kv : span) cyc += (double)(kv.second.second - kv.second.first);
        const uint64_t clk = span.empty() ? 0 : (uint64_t)(cyc / (double)span.size());
        const double ops = (double)blocks * 256.0 * iters * 16.0;
        const double rate = ops / (ms * 1e-3);
        if (rate > best) { best = rate; mhz = (double)clk / (ms * 1e3); }
    }
    cudaFree(dbuf);
    cudaFree(dclk);
    *lop3_per_s = best;
    if (sm_mhz) *sm_mhz = mhz;
    return NSAT_OK;
}

extern "C" int nsat_probe_gather_peak(nsat_ctx* ctx, uint32_t log2_entries, double* gathers_per_s) {
    if (!ctx || !gathers_per_s || log2_entries < 10 || log2_entries > 34) return NSAT_EINVAL;
    if (int rc = set_device(ctx)) return rc;
    const int blocks = ctx->sm_count * 8;
    const uint64_t items = 1ull << 30;
    uint64_t* table = nullptr;
    uint64_t* out = nullptr;
    if (cudaMalloc(&table, (size_t)8 << log2_entries) != cudaSuccess) {
        cudaGetLastError();
        return fail(ctx, NSAT_ENOMEM, "gather probe table does not fit");
    }
    if (cudaMalloc(&out, (size_t)blocks * 256 * 8) != cudaSuccess) {
        cudaGetLastError();
        cudaFree(table);
        return fail(ctx, NSAT_ENOMEM, "gather probe output");
    }
    double best = 0;
    int rc = NSAT_OK;
    if (cudaMemsetAsync(table, 0x5a, (size_t)8 << log2_entries, ctx->stream) != cudaSuccess) rc = NSAT_ECUDA;
    for (int rep = 0; rep < 4 && rc == NSAT_OK; rep++) {
        cudaEventRecord(ctx->ev0[0], ctx->stream);
        if (nsat_launch_gather_probe(table, log2_entries, items, out, blocks, ctx->stream)) { rc = NSAT_ECUDA; break; }
        cudaEventRecord(ctx->ev1[0], ctx->stream);
        if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) { rc = NSAT_ECUDA; break; }
        float ms = 0;
        cudaEventElapsedTime(&ms, ctx->ev0[0], ctx->ev1[0]);
        if (rep > 0 && ms > 0) best = std::max(best, (double)items / (ms * 1e-3));   // rep 0 warms up
    }
    cudaFree(table);
    cudaFree(out);
    if (rc) return fail(ctx, rc, "gather probe failed");
    *gathers_per_s = best;
    return NSAT_OK;
}

// ---------------------------------------------------------------------------
// build check (no device needed)

extern "C" int nsat_jit_check(const nsat_circuit_desc* desc, const uint8_t* quants, int kind,
                              const nsat_opts* opts, nsat_jit_info* info, char* log, size_t loglen) {
    if (!desc || !info || kind < 0 || kind > 2) return NSAT_EINVAL;
    memset(info, 0, sizeof(*info));
    for (uint32_t k = 0; k < desc->gate_num; k++)
        if (desc->gates[3 * k] > 3) return NSAT_EINVAL;
    Circuit c = from_desc(desc);
    if (!c.validate().empty()) return NSAT_EINVAL;
    const bool raw = opts && opts->no_optimize;
    Shape sh;
    sh.block_threads = opts ? opts->block_threads : 0;
    sh.min_blocks = opts ? opts->min_blocks : 0;
    KernelConfig kc;
    std::vector<uint32_t> which{0};
    if (kind == 2) {
        which.clear();
        for (uint32_t j = 0; j < c.outputs.size(); j++) which.push_back(j);
    }
    LutNet net = map_luts_for(c, which, raw, c.n, kCompiledLutWordsPerS);
    std::string err;
    int rc;
    if (kind == 0) {
        SatPlan pl;
        nsat_sat_opts so{};
        so.find_all = 1;
        rc = plan_sat(c.n, so, sh, &pl, &err, (uint32_t)net.luts.size());
        kc = pl.kc;
    } else if (kind == 1) {
        if (!quants) return NSAT_EINVAL;
        std::vector<uint8_t> q(quants, quants + c.n);
        for (auto& v : q) v = v ? 1 : 0;
        QsatPlan pl;
        rc = plan_qsat(c.n, q, false, 0, sh, 0, &pl, &err, (uint32_t)net.luts.size());
        kc = pl.kc;
    } else {
        rc = plan_table(c, false, &kc, &err);
    }
    if (rc) return rc;
    info->lop3_ops = (uint32_t)net.luts.size();
    info->live_gates = net.live_gates;
    std::string src = generate_source(kc, net);
    if (const char* dump = getenv("NSAT_DUMP_DIR")) {   // generated CUDA source, for inspection
        FILE* f = fopen((std::string(dump) + "/jit_check_kind" + std::to_string(kind) + ".cu").c_str(), "w");
        if (f) { fwrite(src.data(), 1, src.size(), f); fclose(f); }
    }
    std::string clog;
    double ms = 0;
    rc = jit_compile_only(src, &clog, &ms, &err);
    info->compile_ms = ms;
    const std::string& text = rc ? err : clog;
    if (log && loglen) {
        size_t k = std::min(loglen - 1, text.size());
        memcpy(log, text.data(), k);
        log[k] = 0;
    }
    if (rc) return NSAT_ECOMPILE;
    // ptxas -v: "Used N registers" and "N bytes spill stores"
    size_t p = clog.find("Used ");
    if (p != std::string::npos) info->regs = atoi(clog.c_str() + p + 5);
    p = clog.find("bytes spill stores");
    if (p != std::string::npos) {
        size_t b = clog.rfind(',', p);
        b = (b == std::string::npos) ? clog.rfind(' ', p - 2) : b + 1;
        info->spill_bytes = atoi(clog.c_str() + b);
    }
    return NSAT_OK;
}

// ---------------------------------------------------------------------------
// autotuning

namespace {

struct Candidate {
    Shape sh;
    double rate = 0;
};

// Assignments per second of the circuit's solve under shape sh: one warm-up
// solve, then solves until sample_ms of device time has accumulated.
int measure_shape(nsat_ctx* ctx, nsat_circuit* c, uint32_t kind, const uint8_t* quants, const Shape& sh,
                  double sample_ms, double* rate) {
    Shape& slot = kind == 0 ? c->tuned : c->tuned_qsat;
    const Shape keep = slot;
    slot = sh;
    if (!slot.block_threads) slot.block_threads = 256;   // an explicit shape, never "unset"
    double dev = 0, items = 0;
    int rc = NSAT_OK;
    for (int run = 0; run < 1000 && rc == NSAT_OK; run++) {
        double ms = 0, it = 0;
        if (kind == 0) {
            nsat_sat_opts o{};
            o.find_all = 1;
            const uint32_t n = c->circ.n;
            const uint32_t bits = std::min<uint32_t>(n, 35);
            const u128 end = (u128)1 << bits;
            o.end_lo = (uint64_t)end;
            o.end_hi = (uint64_t)(end >> 64);
            nsat_sat_result r{};
            rc = nsat_sat_solve(ctx, c, &o, &r);
            ms = r.device_ms;
            it = (double)r.scanned_lo + 18446744073709551616.0 * (double)r.scanned_hi;
        } else {
            // at most 2^35 items: the sub-problem under an all-zero prefix
            nsat_qsat_opts qo{};
            qo.prefix_bits = c->circ.n > 35 ? c->circ.n - 35 : 0;
            nsat_qsat_result r{};
            rc = nsat_qsat_solve(ctx, c, quants, &qo, &r);
            ms = r.device_ms;
            it = (double)r.scanned;
        }
        if (run == 0) continue;      // warm-up: module load, first-launch costs
        dev += ms;
        items += it;
        if (dev >= sample_ms && run >= 2) break;
    }
    slot = keep;
    if (rc) return rc;
    *rate = dev > 0 ? items / (dev * 1e-3) : 0;
    return NSAT_OK;
}

// Compiles the candidates' kernels in parallel host threads (NVRTC is
// thread-safe; modules load into the device's primary context).
void precompile(nsat_ctx* ctx, nsat_circuit* c, uint32_t kind, const std::vector<uint8_t>& q,
                const std::vector<Candidate>& cands, uint32_t threads) {
    std::vector<std::string> srcs;
    const std::vector<uint32_t> out0{0};
    const LutNet& net = get_net(c, out0);
    for (const Candidate& cd : cands) {
        Shape sh = cd.sh;
        if (!sh.block_threads) sh.block_threads = 256;
        std::string err;
        KernelConfig kc;
        if (kind == 0) {
            SatPlan pl;
            nsat_sat_opts o{};
            o.find_all = 1;
            if (plan_sat(c->circ.n, o, sh, &pl, &err, (uint32_t)net.luts.size())) continue;
            kc = pl.kc;
        } else {
            QsatPlan pl;
            if (plan_qsat(c->circ.n, q, false, 0, sh, 0, &pl, &err, (uint32_t)net.luts.size())) continue;
            kc = pl.kc;
        }
        srcs.push_back(generate_source(kc, net));
    }
    const char* name = kind == 0 ? "nsat_sat" : "nsat_qsat";
    const int dev = ctx->device;
    std::atomic<size_t> next{0};
    auto work = [&]() {
        cudaSetDevice(dev);
        cudaFree(nullptr);
        for (size_t i = next++; i < srcs.size(); i = next++) {
            std::shared_ptr<JitModule> m;
            std::string err;
            jit_get(dev, srcs[i], {name}, false, &m, &err);   // failures resurface when measured
        }
    };
    const uint32_t hw = std::max(1u, std::thread::hardware_concurrency());
    const uint32_t nt = std::min<uint32_t>(threads ? threads : hw, (uint32_t)srcs.size());
    std::vector<std::thread> pool;
    for (uint32_t t = 0; t + 1 < nt; t++) pool.emplace_back(work);
    work();
    for (auto& t : pool) t.join();
}

std::string tune_key(nsat_ctx* ctx, nsat_circuit* c, uint32_t kind, const uint8_t* quants) {
    std::string k = "tune2|" + std::to_string(kind) + "|" + std::to_string(c->circ.n) + "|";
    for (const Gate& g : c->circ.gates) k += std::to_string(g.func) + "," + std::to_string(g.i0) + "," + std::to_string(g.i1) + ";";
    k += "|";
    for (const Output& o : c->circ.outputs) k += std::to_string(o.wire) + (o.neg ? "n;" : ";");
    if (kind == 1 && quants)
        for (uint32_t i = 0; i < c->circ.n; i++) k += quants[i] ? 'A' : 'E';
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, ctx->device) == cudaSuccess)
        k += std::string("|") + prop.name + "|" + std::to_string(prop.multiProcessorCount);
    k += "|" + std::to_string(ctx->opts.no_optimize);
    char hex[32];
    snprintf(hex, sizeof(hex), "%016llx", (unsigned long long)jit_fnv(k));
    return jit_cache_dir() + "/tune_" + hex + ".txt";
}

}  // namespace

extern "C" int nsat_autotune(nsat_ctx* ctx, nsat_circuit* c, const nsat_tune_opts* opts, nsat_tune_result* res) {
    if (!ctx || !c || !opts || !res || opts->kind > 1) return NSAT_EINVAL;
    if (opts->kind == 1 && !opts->quants) return NSAT_EINVAL;
    memset(res, 0, sizeof(*res));
    const double t0 = now_ms();
    if (int rc = set_device(ctx)) return rc;
    const uint32_t kind = opts->kind;
    std::vector<uint8_t> q;
    if (kind == 1) {
        q.assign(opts->quants, opts->quants + c->circ.n);
        for (auto& v : q) v = v ? 1 : 0;
    }
    const double sample = opts->sample_ms > 0 ? opts->sample_ms : 60.0;
    Shape& slot = kind == 0 ? c->tuned : c->tuned_qsat;
    const std::string path = tune_key(ctx, c, kind, opts->quants);
    if (opts->persist) {
        FILE* f = fopen(path.c_str(), "r");
        if (f) {
            unsigned bt = 0, mb = 0, cb = 0, sy = 0;
            double rate = 0, drate = 0;
            const int got = fscanf(f, "%u %u %u %u %lf %lf", &bt, &mb, &cb, &sy, &rate, &drate);
            fclose(f);
            if (got == 6 && bt) {
                slot.block_threads = bt; slot.min_blocks = mb; slot.cb_max = cb; slot.sync_every = sy;
                res->block_threads = bt; res->min_blocks = mb; res->cta_bits_max = cb;
                res->sync_every = sync_of(slot);
                res->best_rate = rate; res->default_rate = drate;
                res->from_cache = 1;
                res->tune_ms = now_ms() - t0;
                return NSAT_OK;
            }
        }
    }
    // stage 1: threads per CTA x resident warps per SM (register budget)
    std::vector<Candidate> st1;
    for (uint32_t bt : {128u, 256u, 512u})
        for (uint32_t warps : {16u, 24u, 32u}) {
            Candidate cd;
            cd.sh.block_threads = bt;
            cd.sh.min_blocks = std::max(1u, warps / (bt / 32));
            bool dup = false;
            for (const Candidate& o : st1) dup |= o.sh.block_threads == bt && o.sh.min_blocks == cd.sh.min_blocks;
            if (!dup) st1.push_back(cd);
        }
    precompile(ctx, c, kind, q, st1, opts->threads);
    // the context's own shape: first as a warm-up long enough for the clocks
    // to leave idle (the GPU sat idle while the host compiled), then timed
    const Shape def = effective_shape(ctx, Shape());
    double default_rate = 0, warm = 0;
    if (int rc = measure_shape(ctx, c, kind, opts->quants, def, std::max(250.0, sample), &warm)) return rc;
    if (int rc = measure_shape(ctx, c, kind, opts->quants, def, sample, &default_rate)) return rc;
    Candidate best;
    for (Candidate& cd : st1) {
        if (int rc = measure_shape(ctx, c, kind, opts->quants, cd.sh, sample, &cd.rate)) return rc;
        res->candidates++;
        if (cd.rate > best.rate) best = cd;
    }
    // stage 2: CTA bits per launch (the rest are iterations per warp)
    std::vector<Candidate> st2;
    for (uint32_t cb : {8u, 10u, 14u, 16u}) {
        Candidate cd = best;
        cd.sh.cb_max = cb;
        st2.push_back(cd);
    }
    precompile(ctx, c, kind, q, st2, opts->threads);
    for (Candidate& cd : st2) {
        if (int rc = measure_shape(ctx, c, kind, opts->quants, cd.sh, sample, &cd.rate)) return rc;
        res->candidates++;
        if (cd.rate > best.rate * 1.01) best = cd;     // keep the default CTA cap unless clearly faster
    }
    // stage 3: CTA barrier spacing in the evaluation (instruction-cache sharing)
    std::vector<Candidate> st3;
    for (uint32_t sy : {kNoSync, 32u, 128u}) {
        Candidate cd = best;
        cd.sh.sync_every = sy;
        st3.push_back(cd);
    }
    precompile(ctx, c, kind, q, st3, opts->threads);
    for (Candidate& cd : st3) {
        if (int rc = measure_shape(ctx, c, kind, opts->quants, cd.sh, sample, &cd.rate)) return rc;
        res->candidates++;
        if (cd.rate > best.rate * 1.01) best = cd;
    }
    // the winner and the default once more, back to back
    double again = 0, def_again = 0;
    if (int rc = measure_shape(ctx, c, kind, opts->quants, best.sh, sample, &again)) return rc;
    if (int rc = measure_shape(ctx, c, kind, opts->quants, def, sample, &def_again)) return rc;
    best.rate = std::max(best.rate, again);
    default_rate = std::max(default_rate, def_again);
    if (best.rate < default_rate) {   // the default shape held up
        best.sh = def;
        best.rate = default_rate;
    }
    slot = best.sh;
    if (!slot.block_threads) slot.block_threads = 256;
    if (!slot.cb_max) slot.cb_max = 12;
    res->block_threads = slot.block_threads;
    res->min_blocks = slot.min_blocks;
    res->cta_bits_max = slot.cb_max;
    res->sync_every = sync_of(slot);
    res->best_rate = best.rate;
    res->default_rate = default_rate;
    if (opts->persist) {
        const std::string tmp = path + ".tmp";
        FILE* f = fopen(tmp.c_str(), "w");
        if (f) {
            fprintf(f, "%u %u %u %u %.6e %.6e\n", slot.block_threads, slot.min_blocks, slot.cb_max,
                    slot.sync_every, best.rate, default_rate);
            fclose(f);
            rename(tmp.c_str(), path.c_str());
        }
    }
    res->tune_ms = now_ms() - t0;
    return NSAT_OK;
}

extern "C" int nsat_autotune_reset(nsat_circuit* c) {
    if (!c) return NSAT_EINVAL;
    c->tuned = Shape();
    c->tuned_qsat = Shape();
    return NSAT_OK;
}

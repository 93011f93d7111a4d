// serve.cpp -- batched serving of SAT / QSAT / SATOSTOP jobs on one device.
//
// Jobs are admitted by device memory (a first-fit arena of the server's
// budget), their circuits become LUT bytecode (no compilation), and every
// epoch one CUDA graph runs the interpreter kernel over a slice of tiles of
// every active job: H2D of the epoch's job table, the kernel, D2H of the
// results.  Slices start at one tile (cheap early exits) and double per
// epoch up to a cap, so new arrivals share the device with long jobs right
// away.  Completion rules follow the one-shot solvers:
//   SAT    lowest witness (all lower tiles were evaluated in earlier epochs);
//   QSAT   lowest decisive unit inside tiles, or a host forall/exists reducer
//          over per-tile values for quantifiers above the tile;
//   TABLE  next-state table built tile by tile, then synchronous doubling
//          with step counts (naivesatostop semantics, lowest stopping start).
#include <cuda_runtime.h>

#include <algorithm>
#include <array>
#include <cmath>
#include <atomic>
#include <condition_variable>
#include <mutex>
#include <thread>
#include <chrono>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <set>
#include <string>
#include <vector>

#include "circuit.h"
#include "internal.h"
#include "jit.h"
#include "lutmap.h"
#include "nsat.h"
#include "qreducer.h"
#include "serve_common.h"
#include "serve_kernels.h"
#include "static_kernels.h"

using namespace nsat;

namespace {

constexpr uint32_t kMaxActive = 512;
constexpr uint32_t kDefaultShape = 0;        // index into kSrvShapes when nothing was tuned
constexpr uint64_t kDefaultBudget = 12000000; // epoch budget when nothing was tuned
constexpr size_t kValsCap = 256 * 1024;      // QSAT tile values per epoch
constexpr double kInterpRate = 1.5e12;        // interpreter LUT-words/s (measured), for the tiering estimate

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

uint64_t reverse_bits(uint64_t v, uint32_t bits) {
    uint64_t r = 0;
    for (uint32_t k = 0; k < bits; k++) r |= ((v >> k) & 1ull) << (bits - 1 - k);
    return r;
}

// First-fit allocator over one device allocation (offsets, 256-byte aligned).
struct Arena {
    char* base = nullptr;
    size_t cap = 0, used = 0;
    std::map<size_t, size_t> free_;   // offset -> size
    bool alloc(size_t bytes, size_t* off) {
        bytes = (bytes + 255) & ~(size_t)255;
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second >= bytes) {
                *off = it->first;
                size_t rest = it->second - bytes;
                size_t noff = it->first + bytes;
                free_.erase(it);
                if (rest) free_[noff] = rest;
                used += bytes;
                return true;
            }
        }
        return false;
    }
    void release(size_t off, size_t bytes) {
        bytes = (bytes + 255) & ~(size_t)255;
        used -= bytes;
        auto it = free_.emplace(off, bytes).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) { it->second += nx->second; free_.erase(nx); }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) { pv->second += it->second; free_.erase(it); }
        }
    }
};

// LUT cover of the requested outputs as an interpreter program:
// - scheduled into groups of `group` instructions none of which reads
//   another's result (the kernel loads a whole group's operands before it
//   stores any result): each group takes the lowest-numbered ready LUTs, so
//   the original topological order, and with it the live set, is kept; a NOP
//   on a scratch slot fills a group that finds too few ready LUTs;
// - slot-allocated by liveness over the groups.  Inputs start in slots
//   0..n-1 (the kernel rewrites them every pass), and every slot, an input's
//   included, is reused after the group that reads it last.
struct Program {
    std::vector<SrvIns> ins;
    std::vector<uint16_t> outs;
    uint32_t nslots = 0;
    uint32_t luts = 0;
    uint32_t nops = 0;
};

bool build_program(const Circuit& c, const std::vector<uint32_t>& which, bool raw, uint32_t group, Program* p,
                   std::string* err) {
    LutNet net = map_luts_for(c, which, raw, c.n, kServedLutWordsPerS, true);
    const uint32_t W = c.wires();
    const size_t L = net.luts.size();
    std::vector<int32_t> lut_of(W, -1);
    for (size_t k = 0; k < L; k++) lut_of[net.luts[k].wire] = (int32_t)k;
    auto distinct_in = [&](const Lut& X, int i) {
        for (int j = 0; j < i; j++)
            if (X.in[j] == X.in[i]) return false;
        return true;
    };
    std::vector<std::vector<uint32_t>> users(L);
    std::vector<uint32_t> pending(L, 0);
    for (size_t k = 0; k < L; k++) {
        const Lut& X = net.luts[k];
        for (int i = 0; i < 3; i++) {
            const int32_t q = lut_of[X.in[i]];
            if (q >= 0 && distinct_in(X, i)) { users[q].push_back((uint32_t)k); pending[k]++; }
        }
    }
    // groups of LUT indices (-1: NOP)
    std::set<uint32_t> ready;
    for (size_t k = 0; k < L; k++) if (!pending[k]) ready.insert((uint32_t)k);
    std::vector<std::array<int64_t, SRV_MAX_GROUP>> groups;
    size_t done = 0;
    while (done < L) {
        std::array<int64_t, SRV_MAX_GROUP> grp;
        grp.fill(-1);
        int used = 0;
        while (used < (int)group && !ready.empty()) {
            grp[used++] = *ready.begin();
            ready.erase(ready.begin());
        }
        for (int k = 0; k < used; k++) {
            for (uint32_t u : users[grp[k]]) if (--pending[u] == 0) ready.insert(u);
        }
        p->nops += group - used;
        done += used;
        groups.push_back(grp);
    }
    // slot allocation over the groups
    std::vector<int64_t> last(W, -1);
    for (size_t g = 0; g < groups.size(); g++)
        for (int64_t q : groups[g])
            if (q >= 0) for (int i = 0; i < 3; i++) last[net.luts[q].in[i]] = (int64_t)g;
    for (const Output& o : net.outs) last[o.wire] = INT64_MAX;
    std::vector<int32_t> slot(W, -1);
    for (uint32_t i = 0; i < c.n; i++) slot[i] = (int32_t)i;
    uint32_t next = c.n;
    std::vector<uint32_t> freel;
    for (uint32_t i = c.n; i-- > 0;) if (last[i] < 0) freel.push_back(i);   // unread inputs
    const uint32_t scratch = next++;       // NOP operands and target
    p->ins.clear();
    p->ins.reserve(groups.size() * group);
    for (size_t g = 0; g < groups.size(); g++) {
        // operands read for the last time in this group free their slots first
        for (int64_t q : groups[g]) {
            if (q < 0) continue;
            const Lut& X = net.luts[q];
            for (int i = 0; i < 3; i++) {
                const uint32_t w = X.in[i];
                if (last[w] == (int64_t)g) {
                    freel.push_back((uint32_t)slot[w]);
                    last[w] = -2;   // freed once, however many readers this group has
                }
            }
        }
        for (uint32_t k = 0; k < group; k++) {
            const int64_t q = groups[g][k];
            uint32_t a = scratch, b = scratch, cc = scratch, d = scratch, tt = 0;
            if (q >= 0) {
                const Lut& X = net.luts[q];
                if (!freel.empty()) { d = freel.back(); freel.pop_back(); }
                else d = next++;
                slot[X.wire] = (int32_t)d;
                a = (uint32_t)slot[X.in[0]];
                b = (uint32_t)slot[X.in[1]];
                cc = (uint32_t)slot[X.in[2]];
                tt = X.tt;
            }
            SrvIns r;
            r.ab = a | b << 16;
            r.cd = cc | d << 16;
            r.tlo = r.thi = 0;
            for (int k = 0; k < 4; k++) {
                r.tlo |= ((tt >> k) & 1u) << (8 * k + 7);
                r.thi |= ((tt >> (k + 4)) & 1u) << (8 * k + 7);
            }
            p->ins.push_back(r);
        }
    }
    p->luts = (uint32_t)L;
    p->nslots = next;
    if (next > SRV_MAX_SLOTS) {
        *err = "circuit needs " + std::to_string(next) + " slots, the interpreter holds " +
               std::to_string(SRV_MAX_SLOTS);
        return false;
    }
    p->outs.clear();
    for (const Output& o : net.outs) p->outs.push_back((uint16_t)(slot[o.wire] | (o.neg ? 0x8000 : 0)));
    return true;
}

struct Job {
    uint64_t id = 0, tag = 0;
    uint32_t kind = 0;
    Circuit circ;
    std::vector<uint8_t> quants;
    uint32_t unknowns = 0;
    Program prog;
    uint32_t n = 0, nb = 0, d = 0;   // inputs, enumeration bits, dummy bits
    uint32_t f = 0, m = 0;           // QSAT first block length, unit level
    uint64_t total_tiles = 0;
    uint64_t cursor = 0;             // the device cursor as of the last processed epoch
    uint32_t slot = UINT32_MAX;      // entry of the server's state array
    uint64_t sched = 0;              // tiles handed to launched epochs
    uint64_t slice = 1;
    uint32_t inflight = 0;           // launched epochs holding a slice whose results are not processed yet
    std::unique_ptr<QuantReducer> qr;
    SrvJob rec{};
    size_t prog_off = 0, outs_off = 0, table_off = 0, table2_off = 0, reserve = 0;
    bool any_stop = false;
    bool find_all = false;
    bool finished = false;
    // program build on a builder thread: 0 pending, 1 built, < 0 status code
    std::atomic<int> built{0};
    std::vector<uint32_t> which;     // outputs the program computes
    std::string build_err;
    uint64_t count = 0;
    nsat_job_result res{};
    // QSAT tiering: a compiled kernel races the interpreter (see tier_loop)
    std::atomic<int> tier{0};            // TIER_* below
    std::atomic<bool> tier_cancel{false};
    std::atomic<int64_t> run_from{-1};   // first block the worker solves (set by step)
    double tier_est_ms = 0;              // interpreter estimate for the whole job (queue priority)
    uint32_t tier_s = 0;                 // prefix bits of a block
    uint64_t tier_block = 0;             // tiles per block
    uint64_t stop_at = UINT64_MAX;       // the interpreter stops at this tile
    uint64_t next_block = 0;             // next block result to fold in
    std::mutex tmu;                      // guards blk
    std::condition_variable tcv;         // run_from / cancel for the worker
    std::map<uint64_t, nsat_qsat_result> blk;   // block results by prefix
    int tier_rc = NSAT_OK;
    bool emitted = false;                // result handed to poll, arena memory released
};

enum { TIER_NONE = 0, TIER_COMPILING = 1, TIER_READY = 2, TIER_RUNNING = 3, TIER_DONE = 4 };

// One of the two epoch buffers: while the device runs the epoch of one, the
// host reads the results of the other and fills it again.
struct EpochBuf {
    SrvEpoch* d_hdr = nullptr;
    SrvJob* d_jobs = nullptr;
    uint8_t* d_vals = nullptr;
    SrvEpoch* h_hdr = nullptr;
    SrvJob* h_jobs = nullptr;
    SrvState* h_state = nullptr;     // the state array as the epoch left it
    uint8_t* h_vals = nullptr;
    // epoch graphs by (narrow slots, wide slots; 0 = no wide launch)
    std::map<std::pair<uint32_t, uint32_t>, cudaGraphExec_t> graphs;
    uint32_t max_slots = 0;
    int grid = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::vector<Job*> jobs;          // the launched epoch's jobs, in table order
    bool launched = false;
};

}  // namespace

struct nsat_server {
    nsat_ctx* ctx = nullptr;
    nsat_server_opts opts{};
    Arena arena;
    std::deque<std::unique_ptr<Job>> queue;
    std::vector<std::unique_ptr<Job>> active;
    std::vector<std::unique_ptr<Job>> parked;   // answered jobs a tiering worker still reads
    std::vector<nsat_job_result> done;
    uint64_t next_id = 1;
    uint32_t rr = 0;   // rotating start of the epoch table
    EpochBuf buf[2];
    int cur = 0;       // buffer the next epoch is built in
    cudaStream_t cap = nullptr, cap2 = nullptr;   // streams the epoch graphs are captured on (never run work)
    cudaEvent_t fork = nullptr, join = nullptr;
    SrvState* d_state = nullptr;     // kMaxActive persistent job states (cursor, results)
    SrvState* h_state_init = nullptr;
    std::vector<uint32_t> free_slots;
    NsatJoinState* d_join = nullptr;
    NsatJoinState* h_join = nullptr;
    uint64_t epochs = 0, launches = 0;
    uint64_t launched = 0;   // epochs launched (the sequence number of the last one)
    uint32_t shape = 0;      // interpreter shape (index into kSrvShapes)
    uint64_t h2d_bytes = 0, d2h_bytes = 0;   // host<->device traffic the server issued
    double device_ms = 0;
    // builder threads: programs are built off the caller's thread
    std::mutex bmu;
    std::condition_variable bcv, built_cv;
    std::deque<Job*> bqueue;
    std::vector<std::thread> builders;
    bool stopping = false;
    // QSAT tiering workers, each with its own context on the device
    std::mutex tqmu;
    std::condition_variable tqcv;
    std::deque<Job*> tqueue;
    std::vector<std::thread> tier_workers;
    std::atomic<bool> tstop{false};
    bool tier_enabled = false;

    void stop_tiers() {
        tstop = true;
        {
            std::lock_guard<std::mutex> lk(tqmu);
            for (Job* j : tqueue) j->tier = TIER_DONE;
            tqueue.clear();
        }
        tqcv.notify_all();
        for (auto& t : tier_workers) t.join();
        tier_workers.clear();
    }

    void stop_builders() {
        {
            std::lock_guard<std::mutex> lk(bmu);
            stopping = true;
            bqueue.clear();
        }
        bcv.notify_all();
        for (auto& t : builders) t.join();
        builders.clear();
    }

    ~nsat_server() {
        stop_builders();
        stop_tiers();
        cudaSetDevice(ctx_device(ctx));
        cudaStreamSynchronize(ctx_stream(ctx));
        for (EpochBuf& b : buf) {
            for (auto& kv : b.graphs) cudaGraphExecDestroy(kv.second);
            cudaFree(b.d_hdr);
            cudaFree(b.d_jobs);
            cudaFree(b.d_vals);
            cudaFreeHost(b.h_hdr);
            cudaFreeHost(b.h_jobs);
            cudaFreeHost(b.h_state);
            cudaFreeHost(b.h_vals);
            if (b.ev0) cudaEventDestroy(b.ev0);
            if (b.ev1) cudaEventDestroy(b.ev1);
        }
        if (cap) cudaStreamDestroy(cap);
        if (cap2) cudaStreamDestroy(cap2);
        if (fork) cudaEventDestroy(fork);
        if (join) cudaEventDestroy(join);
        cudaFree(arena.base);
        cudaFree(d_state);
        cudaFreeHost(h_state_init);
        cudaFree(d_join);
        cudaFreeHost(h_join);
    }
};

namespace {

#define SCK(call)                                                                                   \
    do {                                                                                            \
        cudaError_t e_ = (call);                                                                    \
        if (e_ != cudaSuccess)                                                                      \
            return ctx_fail(s->ctx, e_ == cudaErrorMemoryAllocation ? NSAT_ENOMEM : NSAT_ECUDA,      \
                            std::string(#call) + ": " + cudaGetErrorString(e_));                    \
    } while (0)

// Captures buffer b's epoch graph for (narrow, wide) slots per warp: H2D of
// the table; the narrow launch and, when wide > 0, the wide launch as
// parallel branches; D2H of the table and the QSAT tile values.
int capture_graph(nsat_server* s, EpochBuf& b, uint32_t narrow, uint32_t wide, cudaGraphExec_t* out) {
    int per_sm[2] = {0, 0};
    const uint32_t slots[2] = {narrow, wide};
    for (int c = 0; c < (wide ? 2 : 1); c++)
        if (nsat_serve_occupancy(slots[c], s->shape, &per_sm[c]) || per_sm[c] < 1)
            return ctx_fail(s->ctx, NSAT_EUNSUPPORTED, "interpreter does not fit with " + std::to_string(slots[c]) + " slots");
    b.grid = per_sm[0] * ctx_sm_count(s->ctx);
    cudaGraph_t g = nullptr;
    cudaStream_t st = s->cap;
    SCK(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(b.d_hdr, b.h_hdr, sizeof(SrvEpoch), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(b.d_jobs, b.h_jobs, sizeof(SrvJob) * kMaxActive, cudaMemcpyHostToDevice, st);
    int rc = 0;
    if (wide) {
        cudaEventRecord(s->fork, st);
        cudaStreamWaitEvent(s->cap2, s->fork, 0);
        rc |= nsat_launch_serve_epoch(b.d_hdr, b.d_jobs, wide, b.d_vals, per_sm[1] * ctx_sm_count(s->ctx), 1, s->shape,
                                      s->cap2);
        cudaEventRecord(s->join, s->cap2);
    }
    rc |= nsat_launch_serve_epoch(b.d_hdr, b.d_jobs, narrow, b.d_vals, b.grid, 0, s->shape, st);
    if (wide) cudaStreamWaitEvent(st, s->join, 0);
    cudaMemcpyAsync(b.h_state, s->d_state, sizeof(SrvState) * kMaxActive, cudaMemcpyDeviceToHost, st);
    cudaMemcpyAsync(b.h_vals, b.d_vals, kValsCap, cudaMemcpyDeviceToHost, st);
    cudaError_t ce = cudaStreamEndCapture(st, &g);
    if (rc || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        return ctx_fail(s->ctx, NSAT_ECUDA, "epoch graph capture failed");
    }
    cudaError_t ie = cudaGraphInstantiate(out, g, 0);
    cudaGraphDestroy(g);
    if (ie != cudaSuccess) return ctx_fail(s->ctx, NSAT_ECUDA, std::string("cudaGraphInstantiate: ") + cudaGetErrorString(ie));
    b.max_slots = std::max(b.max_slots, std::max(narrow, wide));
    return NSAT_OK;
}

void finish(nsat_server* s, Job* j) {
    j->res.done_ms = now_ms();
    j->res.status = NSAT_OK;
    s->done.push_back(j->res);
}

size_t prog_bytes(const Job* j) { return j->prog.ins.size() * sizeof(SrvIns) + sizeof(SrvIns); }
size_t outs_bytes(const Job* j) { return j->prog.outs.size() * 2 + 2; }
size_t table_bytes(const Job* j) { return j->kind == SRV_TABLE ? ((size_t)8 << j->n) : 0; }

int admit(nsat_server* s, Job* j) {
    const size_t pbytes = prog_bytes(j), obytes = outs_bytes(j), tbytes = table_bytes(j);
    size_t offs[4] = {0, 0, 0, 0};
    const size_t sizes[4] = {pbytes, obytes, tbytes, tbytes};
    const int parts = tbytes ? 4 : 2;
    if (s->free_slots.empty()) return 1;
    for (int i = 0; i < parts; i++) {
        if (!s->arena.alloc(sizes[i], &offs[i])) {
            for (int k = 0; k < i; k++) s->arena.release(offs[k], sizes[k]);
            return 1;
        }
    }
    j->slot = s->free_slots.back();
    s->free_slots.pop_back();
    j->prog_off = offs[0]; j->outs_off = offs[1];
    j->table_off = offs[2]; j->table2_off = offs[3];
    j->reserve = pbytes + obytes + 2 * tbytes;
    cudaStream_t st = ctx_stream(s->ctx);
    // ordered before every epoch that reads them (same stream)
    SCK(cudaMemcpyAsync(s->arena.base + j->prog_off, j->prog.ins.data(), j->prog.ins.size() * sizeof(SrvIns),
                        cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(s->arena.base + j->outs_off, j->prog.outs.data(), j->prog.outs.size() * 2, cudaMemcpyHostToDevice, st));
    SCK(cudaMemcpyAsync(s->d_state + j->slot, s->h_state_init, sizeof(SrvState), cudaMemcpyHostToDevice, st));
    s->h2d_bytes += j->prog.ins.size() * sizeof(SrvIns) + j->prog.outs.size() * 2 + sizeof(SrvState);
    SrvJob& r = j->rec;
    memset(&r, 0, sizeof(r));
    r.prog = (const SrvIns*)(s->arena.base + j->prog_off);
    r.outs = (const uint16_t*)(s->arena.base + j->outs_off);
    r.st = s->d_state + j->slot;
    r.flags = j->find_all ? SRV_JOB_FIND_ALL : 0u;
    r.table = tbytes ? (srv_u64*)(s->arena.base + j->table_off) : nullptr;
    r.ngroups = (uint32_t)(j->prog.ins.size() / kSrvShapes[s->shape].group);
    r.nslots = j->prog.nslots;
    r.kind = j->kind;
    r.nb = j->nb;
    r.nout = (uint32_t)j->prog.outs.size();
    r.m = j->m;
    r.n = j->n;
    for (int p = 0; p < SRV_MAX_NB; p++) r.in_slot[p] = -1;
    if (j->kind == SRV_SAT) {
        for (uint32_t p = j->d; p < j->nb; p++) r.in_slot[p] = (int8_t)(p - j->d);
    } else if (j->kind == SRV_QSAT) {
        for (uint32_t p = 0; p < j->nb; p++) {
            int in = (int)(j->nb - 1 - p);
            if (in < (int)j->n) r.in_slot[p] = (int8_t)in;
        }
        r.q0all = j->quants[0];
        uint64_t ab = 0;
        for (uint32_t p = 0; p < j->nb && p < 64; p++)
            if (j->quants[j->nb - 1 - p]) ab |= 1ull << p;
        r.allbits = ab;
    } else {
        for (uint32_t p = 0; p < j->n; p++) r.in_slot[p] = (int8_t)p;
    }
    j->res.admit_ms = now_ms();
    return 0;
}

void release(nsat_server* s, Job* j) {
    s->free_slots.push_back(j->slot);
    j->slot = UINT32_MAX;
    s->arena.release(j->prog_off, prog_bytes(j));
    s->arena.release(j->outs_off, outs_bytes(j));
    if (j->kind == SRV_TABLE) {
        s->arena.release(j->table_off, table_bytes(j));
        s->arena.release(j->table2_off, table_bytes(j));
    }
}

// Synchronous doubling on a finished table (naivesatostop: lowest stopping
// start, with steps).
int run_joins(nsat_server* s, Job* j) {
    cudaStream_t st = ctx_stream(s->ctx);
    j->res.found = 0;
    if (!j->any_stop) return NSAT_OK;
    NsatJoinState* h = s->h_join;
    memset(h, 0, sizeof(*h));
    for (int i = 0; i < 72; i++) h->best[i] = ~0ull;
    SCK(cudaMemcpyAsync(s->d_join, h, sizeof(*h), cudaMemcpyHostToDevice, st));
    s->h2d_bytes += sizeof(*h);
    s->d2h_bytes += sizeof(*h) + 8;
    void* buf[2] = {s->arena.base + j->table_off, s->arena.base + j->table2_off};
    int src = 0;
    for (uint32_t r = 1; r <= j->n; r++) {
        if (nsat_launch_join_round(2, buf[src], buf[src ^ 1], 1ull << j->n, j->n, j->unknowns, r, 1, s->d_join,
                                   ctx_sm_count(s->ctx), st))
            return ctx_fail(s->ctx, NSAT_ECUDA, "join launch failed");
        s->launches++;
        src ^= 1;
    }
    SCK(cudaMemcpyAsync(h, s->d_join, sizeof(*h), cudaMemcpyDeviceToHost, st));
    SCK(cudaStreamSynchronize(st));
    const uint32_t fr = h->final_round ? h->final_round : j->n;
    const uint64_t best = h->best[fr];
    if (best != ~0ull) {
        uint64_t e = 0;
        SCK(cudaMemcpy(&e, (uint64_t*)buf[fr & 1] + best, 8, cudaMemcpyDeviceToHost));
        j->res.found = 1;
        j->res.start = best;
        j->res.end = e & ((1ull << j->n) - 1);
        j->res.steps = e >> 32;
    }
    return NSAT_OK;
}

}  // namespace

namespace {

// Builder thread: LUT cover, schedule and slot allocation of queued jobs.
void builder_loop(nsat_server* s, bool raw) {
    for (;;) {
        Job* j = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->bmu);
            s->bcv.wait(lk, [s] { return s->stopping || !s->bqueue.empty(); });
            if (s->stopping) return;
            j = s->bqueue.front();
            s->bqueue.pop_front();
        }
        std::string err;
        int st = 1;
        if (!build_program(j->circ, j->which, raw, kSrvShapes[s->shape].group, &j->prog, &err)) {
            st = NSAT_EUNSUPPORTED;
        } else {
            // a job that could never be admitted is answered with an error
            // rather than blocking the queue
            auto round = [](size_t b) { return (b + 255) & ~(size_t)255; };
            const size_t need = round(prog_bytes(j)) + round(outs_bytes(j)) + 2 * round(table_bytes(j));
            if (need > s->arena.cap) {
                st = NSAT_ENOMEM;
                err = "job needs " + std::to_string(need) + " bytes, the server arena holds " + std::to_string(s->arena.cap);
            }
        }
        j->build_err = err;
        // QSAT jobs that would keep the interpreter busy long race a compiled kernel
        if (st == 1 && j->kind == SRV_QSAT && j->d == 0 && j->nb >= SRV_TILE_BITS + 4 && j->nb <= 60 &&
            s->tier_enabled) {
            const double est_ms = std::ldexp(1.0, (int)j->nb - 5) * (double)j->prog.ins.size() / kInterpRate * 1e3;
            if (est_ms > (double)s->opts.tier_min_ms) {
                j->tier_est_ms = est_ms;
                j->tier_s = 4;
                j->tier_block = j->total_tiles >> j->tier_s;
                j->tier = TIER_COMPILING;
                {
                    std::lock_guard<std::mutex> lk(s->tqmu);
                    s->tqueue.push_back(j);
                }
                s->tqcv.notify_one();
            }
        }
        {
            std::lock_guard<std::mutex> lk(s->bmu);
            j->built.store(st, std::memory_order_release);
        }
        s->built_cv.notify_all();
    }
}

// Tiering worker: compiles a QSAT job's kernel for sub-problems under a
// tier_s-input prefix (a warm solve of the last block, whose result is kept),
// reports ready, waits until the server has stopped interpreting at a block
// boundary, then solves the remaining blocks in order, posting each result.
// Blocks are solved by the one-shot QSAT solver on the worker's own context
// and stream, concurrently with the interpreter epochs.
void tier_loop(nsat_server* s, nsat_opts copts) {
    nsat_ctx* wctx = nullptr;
    if (nsat_create(ctx_device(s->ctx), &copts, &wctx) != NSAT_OK) wctx = nullptr;
    for (;;) {
        Job* j = nullptr;
        {
            std::unique_lock<std::mutex> lk(s->tqmu);
            s->tqcv.wait(lk, [s] { return s->tstop.load() || !s->tqueue.empty(); });
            if (s->tstop) break;
            // the largest estimated job first: one compile saves the most interpreter time there
            auto best = s->tqueue.begin();
            for (auto it = s->tqueue.begin(); it != s->tqueue.end(); ++it)
                if ((*it)->tier_est_ms > (*best)->tier_est_ms) best = it;
            j = *best;
            s->tqueue.erase(best);
        }
        if (!wctx || j->tier_cancel) {
            j->tier = TIER_DONE;
            continue;
        }
        const uint32_t sbits = j->tier_s;
        const uint64_t nblocks = 1ull << sbits;
        // the circuit on this worker's context
        std::vector<uint32_t> gates, outs;
        for (const Gate& g : j->circ.gates) { gates.push_back(g.func); gates.push_back(g.i0); gates.push_back(g.i1); }
        for (const Output& o : j->circ.outputs) { outs.push_back(o.wire); outs.push_back(o.neg ? 1 : 0); }
        nsat_circuit_desc desc{j->circ.n, (uint32_t)j->circ.gates.size(), gates.data(),
                               (uint32_t)j->circ.outputs.size(), outs.data()};
        nsat_circuit* cw = nullptr;
        int rc = nsat_circuit_new(wctx, &desc, &cw);
        auto solve = [&](uint64_t p, nsat_qsat_result* r) {
            nsat_qsat_opts qo{};
            qo.prefix_bits = sbits;
            qo.prefix = p;
            return nsat_qsat_solve(wctx, cw, j->quants.data(), &qo, r);
        };
        if (rc == NSAT_OK) {
            nsat_qsat_result r{};
            rc = solve(nblocks - 1, &r);   // compiles and loads the kernel
            if (rc == NSAT_OK) {
                std::lock_guard<std::mutex> lk(j->tmu);
                j->blk[nblocks - 1] = r;
            }
        }
        if (rc != NSAT_OK) {
            j->tier_rc = rc;
            if (cw) nsat_circuit_free(cw);
            j->tier = TIER_DONE;
            continue;
        }
        j->tier = TIER_READY;
        // wait for the handoff (or a cancel)
        int64_t from = -1;
        {
            std::unique_lock<std::mutex> lk(j->tmu);
            while (!j->tier_cancel && !s->tstop && (from = j->run_from.load()) < 0)
                j->tcv.wait_for(lk, std::chrono::milliseconds(50));
        }
        if (from >= 0 && !j->tier_cancel && !s->tstop) {
            j->tier = TIER_RUNNING;
            // the remaining blocks back to back: their launches queue on the
            // worker's stream at once, so they fill the gaps between
            // interpreter epochs instead of taking one gap each
            const uint64_t first = (uint64_t)from, count = nblocks - 1 - first;
            auto post = [&](uint64_t p, const nsat_qsat_result& r) {
                {
                    std::lock_guard<std::mutex> lk(j->tmu);
                    j->blk[p] = r;
                }
                return !(j->tier_cancel || s->tstop);
            };
            if (count > 0) {
                int brc = qsat_solve_blocks(wctx, cw, j->quants.data(), sbits, first, count, post);
                if (brc == NSAT_EUNSUPPORTED) {
                    // blocks of several launches each: one solve per block
                    for (uint64_t p = first; p + 1 < nblocks; p++) {
                        if (j->tier_cancel || s->tstop) break;
                        nsat_qsat_result r{};
                        if (solve(p, &r) != NSAT_OK) {
                            j->tier_rc = NSAT_ECUDA;
                            break;
                        }
                        post(p, r);
                    }
                } else if (brc != NSAT_OK) {
                    j->tier_rc = NSAT_ECUDA;
                }
            }
        }
        nsat_circuit_free(cw);
        j->tier = TIER_DONE;
    }
    if (wctx) nsat_destroy(wctx);
}

}  // namespace

namespace {

std::string tuned_path(nsat_ctx* ctx) {
    std::string k = "serve_tune1|";
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, ctx_device(ctx)) == cudaSuccess)
        k += std::string(prop.name) + "|" + std::to_string(prop.multiProcessorCount);
    char hex[32];
    snprintf(hex, sizeof(hex), "%016llx", (unsigned long long)jit_fnv(k));
    return jit_cache_dir() + "/serve_tune_" + hex + ".txt";
}

bool read_tuned(nsat_ctx* ctx, uint32_t* shape, uint64_t* budget) {
    FILE* f = fopen(tuned_path(ctx).c_str(), "r");
    if (!f) return false;
    unsigned sh = 0;
    unsigned long long b = 0;
    const int got = fscanf(f, "%u %llu", &sh, &b);
    fclose(f);
    if (got != 2 || sh < 1 || sh > SRV_NSHAPES || b == 0) return false;
    *shape = sh;
    *budget = b;
    return true;
}

}  // namespace

extern "C" int nsat_server_create(nsat_ctx* ctx, const nsat_server_opts* opts, nsat_server** out) {
    if (!ctx || !out) return NSAT_EINVAL;
    *out = nullptr;
    std::unique_ptr<nsat_server> sp(new nsat_server());
    nsat_server* s = sp.get();
    s->ctx = ctx;
    if (opts) s->opts = *opts;
    if (!s->opts.arena_bytes) s->opts.arena_bytes = 1ull << 30;
    if (!s->opts.max_active || s->opts.max_active > kMaxActive) s->opts.max_active = kMaxActive;
    if (!s->opts.max_queue) s->opts.max_queue = 1u << 20;
    if (!s->opts.max_slice_tiles) s->opts.max_slice_tiles = 4096;
    // a new job starts with 256 tiles (2^23 assignments, well under a
    // millisecond of interpreter time for the trace's circuits): on the mixed
    // serving trace that measured 663 solves/s and p99 85 ms at 150/s, against
    // 558-590 and 96-100 ms when every job started from one tile
    if (!s->opts.first_slice_tiles) s->opts.first_slice_tiles = 256;
    s->opts.first_slice_tiles = std::min(s->opts.first_slice_tiles, s->opts.max_slice_tiles);
    if (s->opts.shape > SRV_NSHAPES) return ctx_fail(ctx, NSAT_EINVAL, "no such interpreter shape");
    if (!s->opts.shape || !s->opts.epoch_budget) {
        // the tuned choice for this GPU, if one was persisted
        uint32_t shape = 0;
        uint64_t budget = 0;
        if (read_tuned(ctx, &shape, &budget)) {
            if (!s->opts.shape) s->opts.shape = shape;
            if (!s->opts.epoch_budget) s->opts.epoch_budget = budget;
        }
    }
    if (!s->opts.epoch_budget) s->opts.epoch_budget = kDefaultBudget;
    s->shape = s->opts.shape ? s->opts.shape - 1 : kDefaultShape;
    SCK(cudaSetDevice(ctx_device(ctx)));
    SCK(cudaMalloc(&s->arena.base, s->opts.arena_bytes));
    s->arena.cap = s->opts.arena_bytes;
    s->arena.free_[0] = s->opts.arena_bytes;
    for (EpochBuf& b : s->buf) {
        SCK(cudaMalloc(&b.d_hdr, sizeof(SrvEpoch)));
        SCK(cudaMalloc(&b.d_jobs, sizeof(SrvJob) * kMaxActive));
        SCK(cudaMalloc(&b.d_vals, kValsCap));
        SCK(cudaMallocHost(&b.h_hdr, sizeof(SrvEpoch)));
        SCK(cudaMallocHost(&b.h_jobs, sizeof(SrvJob) * kMaxActive));
        SCK(cudaMallocHost(&b.h_state, sizeof(SrvState) * kMaxActive));
        SCK(cudaMallocHost(&b.h_vals, kValsCap));
        memset(b.h_hdr, 0, sizeof(SrvEpoch));
        memset(b.h_jobs, 0, sizeof(SrvJob) * kMaxActive);
        SCK(cudaEventCreate(&b.ev0));
        SCK(cudaEventCreate(&b.ev1));
    }
    SCK(cudaStreamCreateWithFlags(&s->cap, cudaStreamNonBlocking));
    SCK(cudaStreamCreateWithFlags(&s->cap2, cudaStreamNonBlocking));
    SCK(cudaEventCreateWithFlags(&s->fork, cudaEventDisableTiming));
    SCK(cudaEventCreateWithFlags(&s->join, cudaEventDisableTiming));
    SCK(cudaMalloc(&s->d_state, sizeof(SrvState) * kMaxActive));
    SCK(cudaMallocHost(&s->h_state_init, sizeof(SrvState)));
    memset(s->h_state_init, 0, sizeof(SrvState));
    s->h_state_init->min_idx = ~0ull;
    for (uint32_t k = kMaxActive; k-- > 0;) s->free_slots.push_back(k);
    SCK(cudaMalloc(&s->d_join, sizeof(NsatJoinState)));
    SCK(cudaMallocHost(&s->h_join, sizeof(NsatJoinState)));
    // defaults measured on the 10,000-request mixed serving trace: 30 ms and
    // 8 workers took its first 3000 requests from 366 to 609 solves/s; on all
    // of it, 12 workers (the compiles are the limit) reach 517 solves/s
    // against 435 with 8.  Thresholds of 4-15 ms tier more jobs and lower p99
    // on some runs, but cost 3-7 % of solves/s on the whole trace.
    if (s->opts.tier_min_ms == 0) s->opts.tier_min_ms = 30;
    const uint32_t hw_tier = std::max(2u, std::min(12u, std::thread::hardware_concurrency() * 3 / 4));
    const uint32_t ntier =
        s->opts.tier_min_ms == 0xffffffffu ? 0 : (s->opts.tier_threads ? s->opts.tier_threads : hw_tier);
    s->tier_enabled = ntier > 0;
    uint32_t nb = s->opts.build_threads;
    if (!nb) nb = std::max(1u, std::min(8u, std::thread::hardware_concurrency() / 2));
    const bool raw = ctx_no_optimize(ctx);
    for (uint32_t t = 0; t < nb; t++) s->builders.emplace_back(builder_loop, s, raw);
    for (uint32_t t = 0; t < ntier; t++) s->tier_workers.emplace_back(tier_loop, s, ctx_opts(ctx));
    *out = sp.release();
    return NSAT_OK;
}

extern "C" void nsat_server_destroy(nsat_server* s) { delete s; }

extern "C" int nsat_server_submit(nsat_server* s, const nsat_job_desc* jd, uint64_t* id) {
    if (!s || !jd || !id) return NSAT_EINVAL;
    if (s->queue.size() >= s->opts.max_queue) return ctx_fail(s->ctx, NSAT_EBUSY, "serving queue is full");
    if (jd->kind > 2) return NSAT_EINVAL;
    std::unique_ptr<Job> j(new Job());
    j->circ = circuit_from_desc(&jd->circuit);
    for (uint32_t k = 0; k < jd->circuit.gate_num; k++)
        if (jd->circuit.gates[3 * k] > 3) return ctx_fail(s->ctx, NSAT_EINVAL, "bad gate function");
    std::string v = j->circ.validate();
    if (!v.empty()) return ctx_fail(s->ctx, NSAT_EINVAL, v);
    j->kind = jd->kind;
    j->tag = jd->tag;
    j->find_all = (jd->flags & NSAT_JOB_FIND_ALL) != 0;
    j->n = j->circ.n;
    std::vector<uint32_t> which{0};
    if (j->kind == SRV_TABLE) {
        if (j->circ.outputs.size() != j->n + 1) return ctx_fail(s->ctx, NSAT_EINVAL, "SATOSTOP circuit needs n+1 outputs");
        if (j->n > 28 || jd->unknowns > j->n) return ctx_fail(s->ctx, NSAT_EUNSUPPORTED, "served SATOSTOP needs n <= 28");
        which.clear();
        for (uint32_t k = 0; k <= j->n; k++) which.push_back(k);
        j->unknowns = jd->unknowns;
        j->nb = j->n;
        j->total_tiles = j->n > SRV_TILE_BITS ? (1ull << (j->n - SRV_TILE_BITS)) : 1;
    } else {
        const uint32_t d = j->n < SRV_TILE_BITS ? SRV_TILE_BITS - j->n : 0;
        j->d = d;
        j->nb = j->n + d;
        if (j->nb > SRV_MAX_NB) return ctx_fail(s->ctx, NSAT_EUNSUPPORTED, "served jobs need n <= 48");
        j->total_tiles = 1ull << (j->nb - SRV_TILE_BITS);
        if (j->kind == SRV_QSAT) {
            if (!jd->quants) return NSAT_EINVAL;
            j->quants.assign(jd->quants, jd->quants + j->n);
            for (auto& q : j->quants) q = q ? 1 : 0;
            const uint8_t last = j->quants[j->n - 1];
            for (uint32_t k = 0; k < d; k++) j->quants.push_back(last ? 0 : 1);
            uint32_t f = 0;
            while (f < j->n && j->quants[f] == j->quants[0]) f++;
            j->f = f;
            j->m = j->nb - f;
            if (j->m >= SRV_TILE_BITS)
                j->qr.reset(new QuantReducer(std::vector<uint8_t>(j->quants.begin(), j->quants.begin() + (j->nb - SRV_TILE_BITS))));
        }
    }
    j->which = which;
    j->slice = s->opts.first_slice_tiles;
    j->id = s->next_id++;
    j->res.id = j->id;
    j->res.tag = j->tag;
    j->res.kind = j->kind;
    j->res.submit_ms = now_ms();
    *id = j->id;
    Job* jp = j.get();
    s->queue.push_back(std::move(j));
    {
        std::lock_guard<std::mutex> lk(s->bmu);
        s->bqueue.push_back(jp);
    }
    s->bcv.notify_one();
    return NSAT_OK;
}

namespace {

// Fills buffer b with slices of the active jobs (within the work budget) and
// launches its epoch graph.  Slices start where the previous launched slice
// ended, so a job may get a slice while its previous one is still running.
int launch_epoch(nsat_server* s, EpochBuf& b) {
    const uint32_t na = (uint32_t)s->active.size();
    uint64_t budget = s->opts.epoch_budget;
    size_t vals = 0;
    uint32_t k = 0, narrow = 32, wide = 0;
    std::vector<Job*> sel[2];
    std::vector<SrvJob> recs[2];
    for (uint32_t t = 0; t < na; t++) {
        Job* j = s->active[(s->rr + t) % na].get();
        if (j->finished) continue;
        if (s->opts.tier_wait && j->tier.load() == TIER_COMPILING) continue;   // compile first
        const uint64_t lim = std::min<uint64_t>(j->total_tiles, j->stop_at);
        j->sched = std::max(j->sched, j->cursor);     // the device may have rolled over past the plan
        if (j->sched >= lim) continue;
        uint64_t want = std::min<uint64_t>(j->slice, lim - j->sched);
        const uint64_t cost_per_tile = std::max<uint64_t>(1, j->prog.ins.size());
        if (k > 0 && want * cost_per_tile > budget) want = budget / cost_per_tile;
        if (j->kind == SRV_QSAT && j->qr) want = std::min<uint64_t>(want, kValsCap - vals);
        if (want == 0) continue;
        SrvJob& r = j->rec;
        r.tile_begin = j->sched;
        r.tile_end = j->sched + want;
        // SAT and SATOSTOP jobs may go on into the next quarter slice when
        // warps run out of planned work; QSAT jobs keep exact slices (their
        // tile values land at planned offsets, and tiering hands blocks over
        // at planned boundaries)
        r.tile_hard = (j->kind == SRV_QSAT || !s->opts.rollover)
                          ? r.tile_end
                          : std::min<uint64_t>(lim, r.tile_end + std::max<uint64_t>(1, want / 4));
        r.val_off = (uint32_t)vals;
        if (j->kind == SRV_QSAT && j->qr) vals += want;
        budget -= std::min<uint64_t>(budget, want * cost_per_tile);
        k++;
        const uint32_t sl = (j->prog.nslots + 15) & ~15u;
        const int c = sl > SRV_NARROW_SLOTS ? 1 : 0;
        if (c) wide = std::max(wide, sl);
        else narrow = std::max(narrow, sl);
        sel[c].push_back(j);
        recs[c].push_back(r);
        j->sched = r.tile_hard;      // the furthest the device may claim
        j->slice = std::min<uint64_t>(j->slice * 2, s->opts.max_slice_tiles);
        j->inflight++;
    }
    if (na) s->rr = (s->rr + 1) % na;
    b.jobs.clear();
    if (k == 0) return NSAT_OK;
    const uint64_t seq = ++s->launched;
    for (int c = 0; c < 2; c++)
        for (Job* j : sel[c]) {
            if (!j->res.first_epoch) j->res.first_epoch = seq;
            j->res.last_epoch = seq;
            j->res.epochs++;
        }
    // table: narrow jobs, then wide ones
    uint32_t i = 0;
    for (int c = 0; c < 2; c++)
        for (size_t q = 0; q < sel[c].size(); q++) {
            b.h_jobs[i++] = recs[c][q];
            b.jobs.push_back(sel[c][q]);
        }
    b.h_hdr->njobs = k;
    b.h_hdr->n_narrow = (uint32_t)sel[0].size();
    b.h_hdr->hi_mul = 65536;
    b.h_hdr->slot_bytes = srv_slot_bytes(s->shape);
    if (sel[0].empty()) narrow = 16;    // only wide jobs: the narrow launch finds nothing
    cudaGraphExec_t& ge = b.graphs[{narrow, wide}];
    if (!ge) {
        if (int rc = capture_graph(s, b, narrow, wide, &ge)) {
            b.graphs.erase({narrow, wide});
            return rc;
        }
    }
    cudaStream_t st = ctx_stream(s->ctx);
    SCK(cudaEventRecord(b.ev0, st));
    SCK(cudaGraphLaunch(ge, st));
    SCK(cudaEventRecord(b.ev1, st));
    b.launched = true;
    s->launches += wide ? 2 : 1;
    s->h2d_bytes += sizeof(SrvEpoch) + sizeof(SrvJob) * kMaxActive;   // the graph's copies
    s->d2h_bytes += sizeof(SrvState) * kMaxActive + kValsCap;
    return NSAT_OK;
}

// Waits for buffer b's epoch and folds its results into the jobs, in tile
// order (epochs are processed in launch order).
int process_epoch(nsat_server* s, EpochBuf& b) {
    SCK(cudaEventSynchronize(b.ev1));
    float ms = 0;
    SCK(cudaEventElapsedTime(&ms, b.ev0, b.ev1));
    s->device_ms += ms;
    s->epochs++;
    b.launched = false;
    for (size_t i = 0; i < b.jobs.size(); i++) {
        Job* j = b.jobs[i];
        const SrvJob& r = b.h_jobs[i];              // the slice as launched
        const SrvState& st = b.h_state[j->slot];   // cursor and results as the epoch left them
        j->inflight--;
        if (j->finished) continue;   // answered by an earlier epoch; this slice ran ahead
        // every tile below the device cursor has been evaluated: the kernels
        // of this and earlier epochs finished before the state was copied
        const uint64_t got = st.claim - j->cursor;
        j->res.tiles += got;
        j->cursor = st.claim;
        bool finished = false;
        if (j->kind == SRV_SAT) {
            j->count = st.count;
            if (st.min_idx != ~0ull && !j->res.satisfiable) {
                // the lowest witness among tiles below the cursor, hence the lowest of all
                j->res.satisfiable = 1;
                j->res.witness_lo = st.min_idx >> j->d;
                if (!j->find_all) finished = true;
            }
            if (j->cursor == j->total_tiles) finished = true;
            j->res.count = j->count >> j->d;
        } else if (j->kind == SRV_QSAT) {
            j->res.reversed = j->quants[0];
            j->res.solution_bits = j->f;
            if (!j->qr) {
                if (st.min_idx != ~0ull) {
                    j->res.has_solution = 1;
                    j->res.solution = reverse_bits(st.min_idx, j->f);
                    finished = true;
                } else if (j->cursor == j->total_tiles) {
                    finished = true;
                }
            } else {
                // QSAT slices are exact (no roll-over): the slice's tiles, in order
                for (uint64_t t = 0; t < r.tile_end - r.tile_begin && !finished; t++) {
                    j->qr->push(b.h_vals[r.val_off + t] != 0);
                    FinalResult fr;
                    if (j->qr->final_result(&fr)) {
                        j->res.has_solution = fr.has_solution;
                        j->res.solution = fr.has_solution ? fr.solution : 0;
                        finished = true;
                    }
                }
            }
            if (finished) j->res.value = j->res.has_solution ? (j->quants[0] ? 0 : 1) : (j->quants[0] ? 1 : 0);
        } else {
            j->any_stop |= st.any != 0;
            if (j->cursor == j->total_tiles) {
                if (int rc = run_joins(s, j)) return rc;
                finished = true;
            }
        }
        if (finished) j->finished = true;
    }
    b.jobs.clear();
    return NSAT_OK;
}

// The QSAT tiering protocol on the server's side, once per step: when a
// job's compiled kernel is ready, the interpreter stops at the next block
// boundary; once every interpreted tile below it is folded in, the worker
// gets the remaining blocks; their results are folded in block order.  A
// block that holds whole first-block units ends the job when it has a
// decisive unit (its witness completes the prefix); otherwise, and for a
// block inside one unit, the block's value stands for each of its tiles in
// the job's forall/exists reducer (the reduction of equal values is that
// value).
void tier_step(nsat_server* s, Job* j) {
    const int t = j->tier.load();
    if (t == TIER_NONE || j->finished) return;
    const uint64_t B = j->tier_block, nblocks = 1ull << j->tier_s;
    if (t >= TIER_READY && j->stop_at == UINT64_MAX && j->tier_rc == NSAT_OK)
        j->stop_at = (j->sched + B - 1) / B * B;
    if (j->stop_at != UINT64_MAX && j->run_from.load() < 0 && j->cursor == j->stop_at && j->inflight == 0) {
        if (j->stop_at >= j->total_tiles) {
            j->tier_cancel = true;       // the interpreter covered every tile
        } else {
            {
                std::lock_guard<std::mutex> lk(j->tmu);
                j->run_from = (int64_t)(j->stop_at / B);
                j->next_block = j->stop_at / B;
            }
            j->tcv.notify_all();
        }
    }
    if (j->run_from.load() < 0) return;
    for (;;) {
        nsat_qsat_result r{};
        {
            std::lock_guard<std::mutex> lk(j->tmu);
            auto it = j->blk.find(j->next_block);
            if (it == j->blk.end()) break;
            r = it->second;
        }
        const uint64_t p = j->next_block++;
        j->res.compiled_blocks++;
        bool finished = false;
        if (j->tier_s < j->f && r.has_solution) {
            // decisive unit in this block: prefix bits, then the block's own first-block bits
            uint64_t sol = 0;
            for (uint32_t k = 0; k < j->tier_s; k++) sol |= ((p >> (j->tier_s - 1 - k)) & 1ull) << k;
            sol |= r.solution_lo << j->tier_s;
            j->res.has_solution = 1;
            j->res.solution = sol;
            finished = true;
        } else if (j->qr) {
            for (uint64_t k = 0; k < B && !finished; k++) {
                j->qr->push(r.value != 0);
                FinalResult fr;
                if (j->qr->final_result(&fr)) {
                    j->res.has_solution = fr.has_solution;
                    j->res.solution = fr.has_solution ? fr.solution : 0;
                    finished = true;
                }
            }
        }
        if (!finished && j->next_block == nblocks) finished = true;   // no decisive unit anywhere
        if (finished) {
            j->res.reversed = j->quants[0];
            j->res.solution_bits = j->f;
            j->res.value = j->res.has_solution ? (j->quants[0] ? 0 : 1) : (j->quants[0] ? 1 : 0);
            j->finished = true;
            j->tier_cancel = true;
            j->tcv.notify_all();
            break;
        }
    }
}

}  // namespace

extern "C" int nsat_server_step(nsat_server* s, uint32_t* n_active, uint32_t* n_queued) {
    if (!s) return NSAT_EINVAL;
    SCK(cudaSetDevice(ctx_device(s->ctx)));
    // admission in arrival order, by device memory, of jobs whose program is built
    if (s->active.empty() && !s->queue.empty()) {
        // nothing runs: wait (briefly) for the first queued job's program
        std::unique_lock<std::mutex> lk(s->bmu);
        Job* f = s->queue.front().get();
        s->built_cv.wait_for(lk, std::chrono::milliseconds(20),
                             [f] { return f->built.load(std::memory_order_acquire) != 0; });
    }
    while (!s->queue.empty() && s->active.size() < s->opts.max_active) {
        Job* j = s->queue.front().get();
        const int b = j->built.load(std::memory_order_acquire);
        if (b == 0) break;           // still building
        if (b < 0) {                 // cannot be served: answered with its status
            j->res.status = b;
            j->res.done_ms = now_ms();
            s->done.push_back(j->res);
            s->queue.pop_front();
            continue;
        }
        int a = admit(s, j);
        if (a < 0) return a;
        if (a > 0) break;   // does not fit yet
        s->active.push_back(std::move(s->queue.front()));
        s->queue.pop_front();
    }
    // launch the next epoch, then read the previous one while it runs
    EpochBuf& next = s->buf[s->cur];
    EpochBuf& prev = s->buf[s->cur ^ 1];
    if (int rc = launch_epoch(s, next)) return rc;
    if (prev.launched) {
        if (int rc = process_epoch(s, prev)) return rc;
    } else if (next.launched) {
        // nothing was in flight: wait for this epoch now (an idle server answers in one step)
        if (int rc = process_epoch(s, next)) return rc;
        s->cur ^= 1;
    }
    s->cur ^= 1;
    for (auto& jp : s->active)
        if (jp->kind == SRV_QSAT) tier_step(s, jp.get());
    // answer and release finished jobs that no launched epoch still reads; a
    // job a tiering worker still reads is parked until the worker lets go
    std::vector<std::unique_ptr<Job>> keep;
    for (auto& jp : s->active) {
        if (jp->finished && jp->inflight == 0) {
            if (jp->tier.load() != TIER_NONE && !jp->tier_cancel) {
                jp->tier_cancel = true;      // answered by the interpreter first
                jp->tcv.notify_all();
            }
            release(s, jp.get());
            finish(s, jp.get());
            const int t = jp->tier.load();
            if (t != TIER_NONE && t != TIER_DONE) s->parked.push_back(std::move(jp));
        } else {
            keep.push_back(std::move(jp));
        }
    }
    s->active.swap(keep);
    std::vector<std::unique_ptr<Job>> still;
    for (auto& jp : s->parked)
        if (jp->tier.load() != TIER_DONE) still.push_back(std::move(jp));
    s->parked.swap(still);
    if (n_active) *n_active = (uint32_t)s->active.size();
    if (n_queued) *n_queued = (uint32_t)s->queue.size();
    return NSAT_OK;
}

extern "C" int nsat_server_poll(nsat_server* s, nsat_job_result* out, uint32_t cap, uint32_t* n) {
    if (!s || !n || (cap && !out)) return NSAT_EINVAL;
    const uint32_t k = (uint32_t)std::min<size_t>(cap, s->done.size());
    for (uint32_t i = 0; i < k; i++) out[i] = s->done[i];
    s->done.erase(s->done.begin(), s->done.begin() + k);
    *n = k;
    return NSAT_OK;
}

extern "C" int nsat_server_stats(nsat_server* s, nsat_server_stats_t* st) {
    if (!s || !st) return NSAT_EINVAL;
    st->epochs = s->epochs;
    st->device_ms = s->device_ms;
    st->active = (uint32_t)s->active.size();
    st->queued = (uint32_t)s->queue.size();
    st->arena_used = s->arena.used;
    st->arena_bytes = s->arena.cap;
    st->graph_slots = std::max(s->buf[0].max_slots, s->buf[1].max_slots);
    st->grid = (uint32_t)std::max(s->buf[0].grid, s->buf[1].grid);
    st->launches = s->launches;
    st->h2d_bytes = s->h2d_bytes;
    st->d2h_bytes = s->d2h_bytes;
    st->shape = s->shape + 1;
    return NSAT_OK;
}

extern "C" int nsat_server_program_check(const nsat_circuit_desc* cd, uint32_t kind, uint32_t shape, uint64_t seed,
                                         uint32_t* slots, uint32_t* luts, uint32_t* nops) {
    if (!cd || kind > 2 || shape > SRV_NSHAPES) return NSAT_EINVAL;
    const uint32_t G = kSrvShapes[shape ? shape - 1 : kDefaultShape].group;
    Circuit c = circuit_from_desc(cd);
    if (!c.validate().empty()) return NSAT_EINVAL;
    std::vector<uint32_t> which;
    if (kind == SRV_TABLE) for (uint32_t k = 0; k < c.outputs.size(); k++) which.push_back(k);
    else which.push_back(0);
    Program p;
    std::string err;
    if (!build_program(c, which, false, G, &p, &err)) return NSAT_EUNSUPPORTED;
    if (slots) *slots = p.nslots;
    if (luts) *luts = p.luts;
    if (nops) *nops = p.nops;
    uint64_t st = seed;
    auto rnd = [&st]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    // slot values persist across passes, as in the kernel's shared memory
    std::vector<uint64_t> sv(p.nslots, 0);
    for (auto& v : sv) v = rnd();
    for (int pass = 0; pass < 2; pass++) {
        std::vector<uint64_t> wv(c.wires(), 0);
        for (uint32_t i = 0; i < c.n; i++) sv[i] = wv[i] = rnd();
        for (size_t k = 0; k < c.gates.size(); k++) {
            const Gate& g = c.gates[k];
            const uint64_t a = wv[g.i0], b = wv[g.i1];
            wv[c.n + k] = g.func == AND ? (a & b) : g.func == NOR ? ~(a | b) : g.func == NIMPL ? (a & ~b) : (a ^ b);
        }
        for (size_t g0 = 0; g0 < p.ins.size(); g0 += G) {
            uint64_t d[SRV_MAX_GROUP];
            for (uint32_t k = 0; k < G; k++) {
                const SrvIns& r = p.ins[g0 + k];
                const uint64_t a = sv[r.ab & 0xffff], b = sv[r.ab >> 16], cc = sv[r.cd & 0xffff];
                uint64_t y = 0;
                for (int t = 0; t < 8; t++) {
                    const uint64_t sel = ((t & 4) ? a : ~a) & ((t & 2) ? b : ~b) & ((t & 1) ? cc : ~cc);
                    const uint32_t word = t < 4 ? r.tlo : r.thi;
                    y |= sel & (((word >> (8 * (t & 3) + 7)) & 1) ? ~0ull : 0ull);
                }
                d[k] = y;
            }
            for (uint32_t k = 0; k < G; k++) sv[p.ins[g0 + k].cd >> 16] = d[k];
        }
        for (size_t j = 0; j < which.size(); j++) {
            const Output& o = c.outputs[which[j]];
            const uint16_t os = p.outs[j];
            const uint64_t got = sv[os & 0x7fff] ^ ((os & 0x8000) ? ~0ull : 0ull);
            const uint64_t exp = wv[o.wire] ^ (o.neg ? ~0ull : 0ull);
            if (got != exp) return NSAT_EINVAL;
        }
    }
    return NSAT_OK;
}

// ---------------------------------------------------------------------------
// autotuner of the interpreter shape and the epoch budget

namespace {

struct CalJob {
    std::vector<uint32_t> gates, outs;
    uint32_t n = 0;
    uint64_t luts = 0;
};

// Serves every calibration job (SAT, count mode) on a new server with the
// given shape and budget; returns LUT-words evaluated, device ms, wall ms
// and epochs, or a status.
int serve_calibration(nsat_ctx* ctx, const std::vector<CalJob>& jobs, uint32_t shape, uint64_t budget,
                      double* lut_words, double* dev_ms, double* wall_ms, uint64_t* epochs) {
    nsat_server_opts o{};
    o.shape = shape;
    o.epoch_budget = budget;
    o.tier_min_ms = 0xffffffffu;      // the interpreter alone
    nsat_server* s = nullptr;
    if (int rc = nsat_server_create(ctx, &o, &s)) return rc;
    const double t0 = now_ms();
    for (size_t i = 0; i < jobs.size(); i++) {
        nsat_job_desc d{};
        d.kind = SRV_SAT;
        d.circuit = nsat_circuit_desc{jobs[i].n, (uint32_t)(jobs[i].gates.size() / 3), jobs[i].gates.data(), 1,
                                      jobs[i].outs.data()};
        d.tag = i;
        d.flags = NSAT_JOB_FIND_ALL;
        uint64_t id = 0;
        if (int rc = nsat_server_submit(s, &d, &id)) {
            nsat_server_destroy(s);
            return rc;
        }
    }
    std::vector<nsat_job_result> res(jobs.size());
    size_t got = 0;
    *lut_words = 0;
    for (;;) {
        uint32_t active = 0, queued = 0, k = 0;
        if (int rc = nsat_server_step(s, &active, &queued)) {
            nsat_server_destroy(s);
            return rc;
        }
        nsat_server_poll(s, res.data(), (uint32_t)res.size(), &k);
        for (uint32_t i = 0; i < k; i++) {
            if (res[i].status != NSAT_OK) {
                nsat_server_destroy(s);
                return res[i].status;
            }
            *lut_words += (double)res[i].tiles * 1024.0 * (double)jobs[res[i].tag].luts;
        }
        got += k;
        if (got == jobs.size() && active == 0 && queued == 0) break;
    }
    *wall_ms = now_ms() - t0;
    nsat_server_stats_t st{};
    nsat_server_stats(s, &st);
    *dev_ms = st.device_ms;
    *epochs = st.epochs;
    nsat_server_destroy(s);
    return NSAT_OK;
}

}  // namespace

extern "C" int nsat_server_tune(nsat_ctx* ctx, const nsat_serve_tune_opts* opts, nsat_serve_tune_result* res) {
    if (!ctx || !res) return NSAT_EINVAL;
    memset(res, 0, sizeof(*res));
    const double t0 = now_ms();
    nsat_serve_tune_opts o{};
    if (opts) o = *opts;
    if (o.persist && !o.retune) {
        uint32_t shape = 0;
        uint64_t budget = 0;
        if (read_tuned(ctx, &shape, &budget)) {
            res->shape = shape;
            res->epoch_budget = budget;
            res->from_cache = 1;
            res->tune_ms = now_ms() - t0;
            return NSAT_OK;
        }
    }
    // the calibration set: random DAGs of the serving generator, 24-30
    // inputs and 100-4000 gates (log-uniform), large enough that the
    // interpreter, not the epochs' fixed costs, takes the time (about
    // 1e11 LUT-words in all)
    const uint32_t njobs = o.jobs ? o.jobs : 24;
    uint64_t st = o.seed ? o.seed : 0x5E7E5E7Eull;
    auto rnd = [&st]() {
        st += 0x9E3779B97F4A7C15ull;
        uint64_t z = st;
        z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
        z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
        return z ^ (z >> 31);
    };
    std::vector<CalJob> jobs(njobs);
    for (uint32_t i = 0; i < njobs; i++) {
        CalJob& j = jobs[i];
        j.n = 24 + (uint32_t)(rnd() % 7);
        const double u = (double)(rnd() >> 11) / (double)(1ull << 53);
        const uint32_t g = (uint32_t)std::exp(std::log(100.0) + u * (std::log(4000.0) - std::log(100.0)));
        j.gates.assign(3 * g, 0);
        j.outs.assign(2, 0);
        uint32_t gn = 0, on = 0;
        if (nsat_gen_random_dag(rnd(), j.n, g, 64, 1, j.gates.data(), g, j.outs.data(), 1, &gn, &on) != NSAT_OK)
            return NSAT_EINVAL;
        j.gates.resize(3 * gn);
        const nsat_circuit_desc d{j.n, gn, j.gates.data(), 1, j.outs.data()};
        const Circuit c = circuit_from_desc(&d);
        j.luts = map_luts_for(c, {0}, ctx_no_optimize(ctx), c.n, kServedLutWordsPerS, true).luts.size();
    }
    // every shape at the default budget, by device time
    double best = -1;
    for (uint32_t sh = 1; sh <= SRV_NSHAPES; sh++) {
        double lw = 0, dms = 0, wms = 0;
        uint64_t ep = 0;
        if (int rc = serve_calibration(ctx, jobs, sh, kDefaultBudget, &lw, &dms, &wms, &ep)) return rc;
        res->lut_words_per_s[sh - 1] = dms > 0 ? lw / (dms * 1e-3) : 0;
        if (res->lut_words_per_s[sh - 1] > best) {
            best = res->lut_words_per_s[sh - 1];
            res->shape = sh;
        }
    }
    // the epoch budget for that shape, by wall clock.  The calibration set
    // measures throughput, not the latency of arrivals, so the default (1.2e7,
    // the most solves/s at the same p99 on the mixed SAT/QSAT/SATOSTOP serving
    // trace) stays unless another budget is clearly faster (5 %) with epochs
    // under 20 ms.
    static constexpr uint64_t budgets[4] = {6000000, 12000000, 24000000, 48000000};
    constexpr int kDefault = 1;
    static_assert(budgets[kDefault] == kDefaultBudget, "the default budget is a candidate");
    for (int b = 0; b < 4; b++) {
        double lw = 0, dms = 0, wms = 0;
        uint64_t ep = 0;
        if (int rc = serve_calibration(ctx, jobs, res->shape, budgets[b], &lw, &dms, &wms, &ep)) return rc;
        res->budget_solves_per_s[b] = wms > 0 ? njobs / (wms * 1e-3) : 0;
        res->budget_epoch_ms[b] = ep ? wms / (double)ep : 0;
    }
    int pick = kDefault;
    for (int b = 0; b < 4; b++)
        if (res->budget_epoch_ms[b] <= 20.0 && res->budget_solves_per_s[b] > 1.05 * res->budget_solves_per_s[pick])
            pick = b;
    res->epoch_budget = budgets[pick];
    if (o.persist) {
        jit_cache_dir_created();
        const std::string path = tuned_path(ctx), tmp = path + ".tmp";
        FILE* f = fopen(tmp.c_str(), "w");
        if (f) {
            fprintf(f, "%u %llu\n", res->shape, (unsigned long long)res->epoch_budget);
            fclose(f);
            rename(tmp.c_str(), path.c_str());
        }
    }
    res->tune_ms = now_ms() - t0;
    return NSAT_OK;
}

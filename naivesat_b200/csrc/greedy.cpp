// greedy.cpp -- partitioned greedysatostop (greedysatostop -p P [-x PREFIX]),
// drop-in for do_solve_with_cpu_builder_with_partitions
// (greedysatostop.rs:692-837) with the table and the joins on the device.
//
// The whole next-state table is a packed image of (n+1)-bit entries (the
// reference's MemImage/FileImage layout, greedysatostop.rs:308-594).  It
// lives in device memory when it fits next to the work buffers; otherwise in
// pinned host memory, partitions crossing PCIe on a copy stream that
// prefetches the next partition while the current join runs; or, with a file
// prefix, in the temp file PREFIXgreedy_temp_<ns> (the reference's
// FileImage), deleted when the solve returns.  The schedule is the
// reference's, so answers agree for every partition count:
//   first pass: 2^lb chunks (lb = min(log2 P + 2, n - 10)) of entries built
//   in order; no STOP anywhere -> no solution;
//   stage 0..n-1, partition i = 0..P-1: dest = partition i; for j = 0..P-1
//   dest joins partition j as the image holds it now (j < i already updated
//   this stage), or, for j == i, a copy of dest as it is at that point; then
//   the lowest unknown start of dest with STOP is the answer, else dest is
//   written back.
// dest is unpacked to u64 entries for the race-free in-place join; the other
// partitions are read packed by the join's gathers.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include <algorithm>
#include <chrono>
#include <cstring>
#include <string>
#include <vector>

#include "greedy_kernels.h"
#include "internal.h"
#include "nsat.h"

using namespace nsat;

namespace {

enum Storage { DEVICE = 0, HOST = 1, FILEIMG = 2 };

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

bool pread_all(int fd, void* buf, uint64_t len, uint64_t off) {
    char* p = static_cast<char*>(buf);
    while (len) {
        const ssize_t r = pread(fd, p, len, (off_t)off);
        if (r <= 0) return false;
        p += r; len -= (uint64_t)r; off += (uint64_t)r;
    }
    return true;
}

bool pwrite_all(int fd, const void* buf, uint64_t len, uint64_t off) {
    const char* p = static_cast<const char*>(buf);
    while (len) {
        const ssize_t r = pwrite(fd, p, len, (off_t)off);
        if (r <= 0) return false;
        p += r; len -= (uint64_t)r; off += (uint64_t)r;
    }
    return true;
}

// Packed bytes of `count` entries of `bits` bits (count a multiple of 64).
uint64_t packed_bytes(uint64_t count, uint32_t bits) { return ((count * bits) >> 6) * 8; }

// The image and every buffer the solve uses.  Device buffers come from the
// context's stream-ordered pool (ctx_alloc), so a repeated solve reuses them.
struct Work {
    nsat_ctx* ctx = nullptr;
    int storage = DEVICE;
    uint64_t bytes = 0;
    uint64_t* dev_image = nullptr;    // DEVICE
    uint64_t* host_image = nullptr;   // HOST (pinned)
    int fd = -1;                      // FILEIMG
    std::string path;
    uint64_t* host_stage = nullptr;   // FILEIMG: pinned staging of one partition or chunk
    uint64_t* dest = nullptr;         // unpacked partition i
    uint64_t* snap = nullptr;         // unpacked copy of dest (j == i)
    uint64_t* stage[2] = {nullptr, nullptr};   // HOST/FILEIMG: packed partitions on the device
    uint64_t* chunk = nullptr;        // first pass: u64 entries of one chunk
    uint64_t* best = nullptr;
    cudaStream_t copy = nullptr;
    cudaEvent_t ready[2] = {nullptr, nullptr}, used[2] = {nullptr, nullptr};
    cudaEvent_t wb = nullptr;
    std::vector<cudaEvent_t> jev;     // a start/end pair per join of one partition step

    ~Work() {
        if (copy) cudaStreamSynchronize(copy);   // the copy stream's uses end before the frees
        if (ctx) {
            for (void* p : {(void*)dev_image, (void*)dest, (void*)snap, (void*)stage[0], (void*)stage[1],
                            (void*)chunk, (void*)best})
                ctx_free(ctx, p);
        }
        if (host_image) cudaFreeHost(host_image);
        if (host_stage) cudaFreeHost(host_stage);
        for (int k = 0; k < 2; k++) {
            if (ready[k]) cudaEventDestroy(ready[k]);
            if (used[k]) cudaEventDestroy(used[k]);
        }
        for (cudaEvent_t e : jev) cudaEventDestroy(e);
        if (wb) cudaEventDestroy(wb);
        if (copy) cudaStreamDestroy(copy);
        if (fd >= 0) close(fd);
        if (!path.empty()) unlink(path.c_str());
    }
};

#define GCK(call)                                                                                 \
    do {                                                                                          \
        cudaError_t e_ = (call);                                                                  \
        if (e_ != cudaSuccess)                                                                    \
            return ctx_fail(ctx, e_ == cudaErrorMemoryAllocation ? NSAT_ENOMEM : NSAT_ECUDA,       \
                            std::string(#call) + ": " + cudaGetErrorString(e_));                  \
    } while (0)

#define KCK(call)                                                                                 \
    do {                                                                                          \
        if ((call) != 0) return ctx_fail(ctx, NSAT_ECUDA, std::string(#call) + " failed");         \
    } while (0)

int check_opts(nsat_ctx* ctx, uint32_t n, const nsat_greedy_opts* o, uint32_t* pbits) {
    const uint32_t P = o->partitions;
    if (P < 2 || (P & (P - 1))) return ctx_fail(ctx, NSAT_EINVAL, "partitions must be a power of two >= 2");
    if (n < 11) return ctx_fail(ctx, NSAT_EUNSUPPORTED, "partitioned solve needs n >= 11");
    if ((uint64_t)P * 64 > (1ull << n)) return ctx_fail(ctx, NSAT_EINVAL, "more partitions than 2^n / 64");
    if (o->unknowns > n) return ctx_fail(ctx, NSAT_EINVAL, "unknowns must not exceed the state length");
    uint32_t b = 0;
    while ((1u << b) < P) b++;
    *pbits = b;
    return NSAT_OK;
}

// Chooses where the image lives and allocates the image and work buffers.
int setup(nsat_ctx* ctx, Work& w, uint32_t n, uint64_t L, uint64_t chunk, const nsat_greedy_opts* o,
          bool joins) {
    w.ctx = ctx;
    const uint32_t P = o->partitions;
    const uint32_t bits = n + 1;
    w.bytes = packed_bytes(1ull << n, bits);
    const uint64_t pbytes = packed_bytes(L, bits), cbytes = packed_bytes(chunk, bits);
    const uint64_t work_dev = (joins ? 2 * L * 8 : 0) + chunk * 8 + 64;
    if (o->file_prefix) {
        w.storage = FILEIMG;
    } else {
        uint64_t budget = o->device_bytes;
        if (!budget) {
            // free device memory less 1 GiB; if the image does not fit, what
            // the context's pool keeps for reuse is returned and counted too
            size_t fr = 0, tot = 0;
            GCK(cudaMemGetInfo(&fr, &tot));
            budget = fr > (1ull << 30) ? fr - (1ull << 30) : 0;
            if (w.bytes + work_dev > budget) {
                ctx_trim(ctx);
                GCK(cudaMemGetInfo(&fr, &tot));
                budget = fr > (1ull << 30) ? fr - (1ull << 30) : 0;
            }
        }
        w.storage = (w.bytes + work_dev <= budget) ? DEVICE : HOST;
    }
    if (w.storage == DEVICE) {
        GCK(ctx_alloc(ctx, (void**)&w.dev_image, w.bytes));
    } else {
        for (int k = 0; k < 2; k++) GCK(ctx_alloc(ctx, (void**)&w.stage[k], std::max(pbytes, cbytes)));
        if (w.storage == HOST) {
            cudaError_t e = cudaMallocHost(&w.host_image, w.bytes);
            if (e != cudaSuccess) {
                w.host_image = nullptr;
                return ctx_fail(ctx, NSAT_ENOMEM, "pinned host image of " + std::to_string(w.bytes) + " bytes: " +
                                                      cudaGetErrorString(e));
            }
        } else {
            const long long ns = (long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
                                     std::chrono::system_clock::now().time_since_epoch()).count();
            w.path = std::string(o->file_prefix) + "greedy_temp_" + std::to_string(ns);
            w.fd = open(w.path.c_str(), O_RDWR | O_CREAT | O_TRUNC, 0600);
            if (w.fd < 0) {
                const std::string p = w.path;
                w.path.clear();
                return ctx_fail(ctx, NSAT_EINVAL, "cannot create image file " + p);
            }
            if (ftruncate(w.fd, (off_t)w.bytes) != 0) return ctx_fail(ctx, NSAT_ENOMEM, "cannot size image file");
            GCK(cudaMallocHost(&w.host_stage, std::max(pbytes, cbytes)));
        }
    }
    GCK(ctx_alloc(ctx, (void**)&w.chunk, chunk * 8));
    GCK(ctx_alloc(ctx, (void**)&w.best, 8));
    if (joins) {
        GCK(ctx_alloc(ctx, (void**)&w.dest, L * 8));
        GCK(ctx_alloc(ctx, (void**)&w.snap, L * 8));
    }
    GCK(cudaStreamSynchronize(ctx_stream(ctx)));   // the pool's buffers are ready on every stream
    GCK(cudaStreamCreateWithFlags(&w.copy, cudaStreamNonBlocking));
    for (int k = 0; k < 2; k++) {
        GCK(cudaEventCreateWithFlags(&w.ready[k], cudaEventDisableTiming));
        GCK(cudaEventCreateWithFlags(&w.used[k], cudaEventDisableTiming));
    }
    GCK(cudaEventCreateWithFlags(&w.wb, cudaEventDisableTiming));
    if (joins) {
        w.jev.assign(2 * P, nullptr);
        for (auto& e : w.jev) GCK(cudaEventCreate(&e));
    }
    return NSAT_OK;
}

// Packed range of the image at byte offset off -> device buffer dst, on
// stream st.  HOST: async from pinned memory; FILEIMG: through the pinned
// staging buffer (synchronous, the staging buffer is reused next).
int fetch(nsat_ctx* ctx, Work& w, uint64_t off, uint64_t len, void* dst, cudaStream_t st, nsat_greedy_result* r) {
    if (w.storage == HOST) {
        GCK(cudaMemcpyAsync(dst, reinterpret_cast<char*>(w.host_image) + off, len, cudaMemcpyHostToDevice, st));
    } else {
        if (!pread_all(w.fd, w.host_stage, len, off)) return ctx_fail(ctx, NSAT_EINVAL, "image file read failed");
        GCK(cudaMemcpyAsync(dst, w.host_stage, len, cudaMemcpyHostToDevice, st));
        GCK(cudaStreamSynchronize(st));
    }
    r->h2d_bytes += len;
    return NSAT_OK;
}

int store(nsat_ctx* ctx, Work& w, uint64_t off, uint64_t len, const void* src, cudaStream_t st,
          nsat_greedy_result* r) {
    if (w.storage == HOST) {
        GCK(cudaMemcpyAsync(reinterpret_cast<char*>(w.host_image) + off, src, len, cudaMemcpyDeviceToHost, st));
    } else {
        GCK(cudaMemcpyAsync(w.host_stage, src, len, cudaMemcpyDeviceToHost, st));
        GCK(cudaStreamSynchronize(st));
        if (!pwrite_all(w.fd, w.host_stage, len, off)) return ctx_fail(ctx, NSAT_EINVAL, "image file write failed");
    }
    r->d2h_bytes += len;
    return NSAT_OK;
}

// First pass: every chunk of entries, packed, into the image in order.
int build_image(nsat_ctx* ctx, nsat_circuit* c, Work& w, uint32_t lb, bool* any_stop, nsat_greedy_result* r) {
    const uint32_t n = circuit_of(c).n, bits = n + 1;
    const uint64_t chunk = 1ull << (n - lb);
    const uint64_t cbytes = packed_bytes(chunk, bits);
    cudaStream_t st = ctx_stream(ctx);
    const int sms = ctx_sm_count(ctx);
    *any_stop = false;
    for (uint64_t a = 0; a < (1ull << lb); a++) {
        uint32_t stop = 0;
        float ms = 0;
        if (int rc = table_chunk_u64(ctx, c, a * chunk, chunk, w.chunk, &stop, &ms)) return rc;
        r->build_ms += ms;
        *any_stop |= stop != 0;
        if (w.storage == DEVICE) {
            KCK(nsat_greedy_pack(w.chunk, chunk, bits, w.dev_image + a * (cbytes / 8), sms, st));
        } else {
            KCK(nsat_greedy_pack(w.chunk, chunk, bits, w.stage[0], sms, st));
            if (int rc = store(ctx, w, a * cbytes, cbytes, w.stage[0], st, r)) return rc;
            GCK(cudaStreamSynchronize(st));   // stage[0] is packed into again next
        }
    }
    GCK(cudaStreamSynchronize(st));
    return NSAT_OK;
}

// One stage step for partition i: dest = partition i joined with every
// partition in order.  HOST images prefetch partition j+1 on the copy stream
// while partition j is joined.
int join_partition(nsat_ctx* ctx, Work& w, uint32_t n, uint32_t P, uint64_t L, uint32_t i, nsat_greedy_result* r) {
    const uint32_t bits = n + 1;
    const uint64_t pbytes = packed_bytes(L, bits), pwords = pbytes / 8;
    cudaStream_t st = ctx_stream(ctx);
    const int sms = ctx_sm_count(ctx);
    // dest
    if (w.storage == DEVICE) {
        KCK(nsat_greedy_unpack(w.dev_image + (uint64_t)i * pwords, L, bits, w.dest, sms, st));
    } else {
        if (int rc = fetch(ctx, w, (uint64_t)i * pbytes, pbytes, w.stage[0], st, r)) return rc;
        KCK(nsat_greedy_unpack(w.stage[0], L, bits, w.dest, sms, st));
    }
    // the partitions other than i, in order; HOST: double-buffered prefetch
    std::vector<uint32_t> others;
    for (uint32_t j = 0; j < P; j++)
        if (j != i) others.push_back(j);
    if (w.storage == HOST) {
        // the copy stream waits for everything issued so far (the write-back
        // of earlier partitions of this stage and dest's own staging)
        GCK(cudaEventRecord(w.wb, st));
        GCK(cudaStreamWaitEvent(w.copy, w.wb, 0));
        GCK(cudaMemcpyAsync(w.stage[0], reinterpret_cast<char*>(w.host_image) + (uint64_t)others[0] * pbytes, pbytes,
                            cudaMemcpyHostToDevice, w.copy));
        GCK(cudaEventRecord(w.ready[0], w.copy));
        r->h2d_bytes += pbytes;
    }
    size_t k = 0;   // next entry of `others`
    for (uint32_t j = 0; j < P; j++) {
        const uint64_t* src = nullptr;
        bool packed = true;
        int slot = (int)(k & 1);
        if (j == i) {
            GCK(cudaMemcpyAsync(w.snap, w.dest, L * 8, cudaMemcpyDeviceToDevice, st));
            src = w.snap;
            packed = false;
        } else if (w.storage == DEVICE) {
            src = w.dev_image + (uint64_t)j * pwords;
        } else if (w.storage == HOST) {
            GCK(cudaStreamWaitEvent(st, w.ready[slot], 0));
            src = w.stage[slot];
            if (k + 1 < others.size()) {
                const int ns = slot ^ 1;
                if (k >= 1) GCK(cudaStreamWaitEvent(w.copy, w.used[ns], 0));   // its last join is done
                GCK(cudaMemcpyAsync(w.stage[ns], reinterpret_cast<char*>(w.host_image) + (uint64_t)others[k + 1] * pbytes,
                                    pbytes, cudaMemcpyHostToDevice, w.copy));
                GCK(cudaEventRecord(w.ready[ns], w.copy));
                r->h2d_bytes += pbytes;
            }
        } else {
            if (int rc = fetch(ctx, w, (uint64_t)j * pbytes, pbytes, w.stage[0], st, r)) return rc;
            src = w.stage[0];
        }
        GCK(cudaEventRecord(w.jev[2 * j], st));
        if (packed) KCK(nsat_greedy_join_packed(w.dest, L, src, (uint64_t)j * L, L, n, sms, st));
        else KCK(nsat_greedy_join(w.dest, L, src, (uint64_t)j * L, L, n, sms, st));
        GCK(cudaEventRecord(w.jev[2 * j + 1], st));
        if (j != i && w.storage == HOST) GCK(cudaEventRecord(w.used[slot], st));
        if (j != i) k++;
        r->joins++;
    }
    // join kernel time (each pair brackets one launch)
    GCK(cudaEventSynchronize(w.jev[2 * P - 1]));
    for (uint32_t j = 0; j < P; j++) {
        float ms = 0;
        GCK(cudaEventElapsedTime(&ms, w.jev[2 * j], w.jev[2 * j + 1]));
        r->join_ms += ms;
    }
    return NSAT_OK;
}

}  // namespace

extern "C" int nsat_greedy_solve(nsat_ctx* ctx, nsat_circuit* c, const nsat_greedy_opts* o, nsat_greedy_result* r) {
    if (!ctx || !c || !o || !r) return NSAT_EINVAL;
    memset(r, 0, sizeof(*r));
    const double t0 = now_ms();
    const Circuit& circ = circuit_of(c);
    const uint32_t n = circ.n, bits = n + 1;
    if (circ.outputs.size() != n + 1) return ctx_fail(ctx, NSAT_EINVAL, "SATOSTOP circuit needs n+1 outputs");
    uint32_t pbits = 0;
    if (int rc = check_opts(ctx, n, o, &pbits)) return rc;
    const uint32_t P = o->partitions;
    const uint32_t lb = std::min(pbits + 2, n - 10);
    r->load_bits = lb;
    const uint64_t L = 1ull << (n - pbits);          // entries per partition
    const uint64_t chunk = 1ull << (n - lb);
    const uint64_t pbytes = packed_bytes(L, bits), pwords = pbytes / 8;
    GCK(cudaSetDevice(ctx_device(ctx)));
    Work w;
    if (int rc = setup(ctx, w, n, L, chunk, o, true)) return rc;
    r->storage = (uint32_t)w.storage;
    bool any_stop = false;
    if (int rc = build_image(ctx, c, w, lb, &any_stop, r)) return rc;
    if (!any_stop) {
        r->wall_ms = now_ms() - t0;
        return NSAT_OK;
    }
    cudaStream_t st = ctx_stream(ctx);
    const int sms = ctx_sm_count(ctx);
    for (uint32_t stage = 0; stage < n; stage++) {
        for (uint32_t i = 0; i < P; i++) {
            const uint64_t start_i = (uint64_t)i * L;
            if (int rc = join_partition(ctx, w, n, P, L, i, r)) return rc;
            uint64_t best = ~0ull;
            GCK(cudaMemcpyAsync(w.best, &best, 8, cudaMemcpyHostToDevice, st));
            KCK(nsat_greedy_find(w.dest, start_i, L, n, o->unknowns, w.best, sms, st));
            GCK(cudaMemcpyAsync(&best, w.best, 8, cudaMemcpyDeviceToHost, st));
            GCK(cudaStreamSynchronize(st));
            if (best != ~0ull) {
                uint64_t e = 0;
                GCK(cudaMemcpy(&e, w.dest + (best - start_i), 8, cudaMemcpyDeviceToHost));
                r->found = 1;
                r->start = best;
                r->end = e & ((1ull << n) - 1);
                r->stage = stage;
                r->partition = i;
                r->wall_ms = now_ms() - t0;
                return NSAT_OK;
            }
            // write dest back to partition i of the image; in device memory the
            // next step's kernels follow in stream order, with no host wait
            if (w.storage == DEVICE) {
                KCK(nsat_greedy_pack(w.dest, L, bits, w.dev_image + (uint64_t)i * pwords, sms, st));
            } else {
                KCK(nsat_greedy_pack(w.dest, L, bits, w.stage[0], sms, st));
                if (int rc = store(ctx, w, (uint64_t)i * pbytes, pbytes, w.stage[0], st, r)) return rc;
                GCK(cudaStreamSynchronize(st));
            }
        }
    }
    GCK(cudaStreamSynchronize(st));   // the last write-back
    r->wall_ms = now_ms() - t0;
    return NSAT_OK;
}

extern "C" int nsat_greedy_image(nsat_ctx* ctx, nsat_circuit* c, uint32_t partitions, const char* file_prefix,
                                 uint64_t* words, uint64_t nwords) {
    if (!ctx || !c || !words) return NSAT_EINVAL;
    const Circuit& circ = circuit_of(c);
    const uint32_t n = circ.n, bits = n + 1;
    if (circ.outputs.size() != n + 1) return ctx_fail(ctx, NSAT_EINVAL, "SATOSTOP circuit needs n+1 outputs");
    nsat_greedy_opts o{};
    o.partitions = partitions;
    o.file_prefix = file_prefix;
    o.device_bytes = file_prefix ? 0 : 1;   // a host image unless a file is asked for
    uint32_t pbits = 0;
    if (int rc = check_opts(ctx, n, &o, &pbits)) return rc;
    const uint64_t total = packed_bytes(1ull << n, bits);
    if (nwords * 8 < total) return ctx_fail(ctx, NSAT_EINVAL, "image buffer too small");
    const uint32_t lb = std::min(pbits + 2, n - 10);
    const uint64_t L = 1ull << (n - pbits), chunk = 1ull << (n - lb);
    GCK(cudaSetDevice(ctx_device(ctx)));
    Work w;
    if (int rc = setup(ctx, w, n, L, chunk, &o, false)) return rc;
    nsat_greedy_result r{};
    bool any = false;
    if (int rc = build_image(ctx, c, w, lb, &any, &r)) return rc;
    if (w.storage == HOST) {
        memcpy(words, w.host_image, total);
    } else if (!pread_all(w.fd, words, total, 0)) {
        return ctx_fail(ctx, NSAT_EINVAL, "image file read failed");
    }
    return NSAT_OK;
}

// greedy.cpp -- partitioned greedysatostop (greedysatostop -p P [-x PREFIX]),
// drop-in for do_solve_with_cpu_builder_with_partitions
// (greedysatostop.rs:692-837) with the table and the joins on the device.
//
// The whole next-state table lives in a packed image of (n+1)-bit entries
// (the reference's MemImage/FileImage layout, greedysatostop.rs:308-594):
// in pinned host memory, or, with a file prefix, in the temp file
// PREFIXgreedy_temp_<ns> that is deleted when the solve returns (the
// reference's FileImage).  The schedule is the reference's, so answers agree
// for every partition count:
//   first pass: 2^lb chunks (lb = min(log2 P + 2, n - 10)) of entries built
//   in order; no STOP anywhere -> no solution;
//   stage 0..n-1, partition i = 0..P-1: dest = partition i; for j = 0..P-1
//   dest joins partition j as the image holds it now (j < i already updated
//   this stage), or, for j == i, a copy of dest as it is at that point; then
//   the lowest unknown start of dest with STOP is the answer, else dest is
//   written back.
// Device memory: two unpacked partitions (dest, second), one packed partition
// and one chunk of the first pass.
#include <cuda_runtime.h>
#include <fcntl.h>
#include <unistd.h>

#include <chrono>
#include <cstring>
#include <string>

#include "greedy_kernels.h"
#include "internal.h"
#include "nsat.h"

using namespace nsat;

namespace {

double now_ms() {
    return std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// Where the packed image lives: pinned host memory or a temp file.
struct Image {
    uint64_t bytes = 0;
    uint64_t* host = nullptr;      // pinned, whole image (no file)
    int fd = -1;
    std::string path;
    uint64_t* stage = nullptr;     // pinned staging for the file case (one partition or chunk)
    uint64_t stage_bytes = 0;

    ~Image() {
        if (host) cudaFreeHost(host);
        if (stage) cudaFreeHost(stage);
        if (fd >= 0) close(fd);
        if (!path.empty()) unlink(path.c_str());
    }
};

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

struct DevBufs {
    uint64_t* dest = nullptr;
    uint64_t* second = nullptr;
    uint64_t* packed = nullptr;
    uint64_t* chunk = nullptr;
    uint64_t* best = nullptr;
    ~DevBufs() {
        cudaFree(dest);
        cudaFree(second);
        cudaFree(packed);
        cudaFree(chunk);
        cudaFree(best);
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

// Packed bytes of `count` entries of `bits` bits (count a multiple of 64).
uint64_t packed_bytes(uint64_t count, uint32_t bits) { return ((count * bits) >> 6) * 8; }

// Copies a packed range of the image (byte offset off, len bytes) to the
// device, through the staging buffer in the file case.
int image_to_device(nsat_ctx* ctx, Image& im, uint64_t off, uint64_t len, void* dev, cudaStream_t st,
                    nsat_greedy_result* r) {
    if (im.host) {
        GCK(cudaMemcpyAsync(dev, reinterpret_cast<char*>(im.host) + off, len, cudaMemcpyHostToDevice, st));
    } else {
        if (!pread_all(im.fd, im.stage, len, off)) return ctx_fail(ctx, NSAT_EINVAL, "image file read failed");
        GCK(cudaMemcpyAsync(dev, im.stage, len, cudaMemcpyHostToDevice, st));
        GCK(cudaStreamSynchronize(st));   // the staging buffer is reused next
    }
    r->h2d_bytes += len;
    return NSAT_OK;
}

int device_to_image(nsat_ctx* ctx, Image& im, uint64_t off, uint64_t len, const void* dev, cudaStream_t st,
                    nsat_greedy_result* r) {
    if (im.host) {
        GCK(cudaMemcpyAsync(reinterpret_cast<char*>(im.host) + off, dev, len, cudaMemcpyDeviceToHost, st));
    } else {
        GCK(cudaMemcpyAsync(im.stage, dev, len, cudaMemcpyDeviceToHost, st));
        GCK(cudaStreamSynchronize(st));
        if (!pwrite_all(im.fd, im.stage, len, off)) return ctx_fail(ctx, NSAT_EINVAL, "image file write failed");
    }
    r->d2h_bytes += len;
    return NSAT_OK;
}

// First pass: every chunk of entries, packed, into the image in order.
int build_image(nsat_ctx* ctx, nsat_circuit* c, Image& im, DevBufs& d, uint32_t lb, bool* any_stop,
                nsat_greedy_result* r) {
    const uint32_t n = circuit_of(c).n, bits = n + 1;
    const uint64_t chunk = 1ull << (n - lb);
    const uint64_t cbytes = packed_bytes(chunk, bits);
    cudaStream_t st = ctx_stream(ctx);
    const int sms = ctx_sm_count(ctx);
    *any_stop = false;
    for (uint64_t a = 0; a < (1ull << lb); a++) {
        uint32_t stop = 0;
        float ms = 0;
        if (int rc = table_chunk_u64(ctx, c, a * chunk, chunk, d.chunk, &stop, &ms)) return rc;
        r->build_ms += ms;
        *any_stop |= stop != 0;
        KCK(nsat_greedy_pack(d.chunk, chunk, bits, d.packed, sms, st));
        if (int rc = device_to_image(ctx, im, a * cbytes, cbytes, d.packed, st, r)) return rc;
    }
    return cudaStreamSynchronize(st) == cudaSuccess ? NSAT_OK : ctx_fail(ctx, NSAT_ECUDA, "first pass failed");
}

int open_image(nsat_ctx* ctx, Image& im, uint64_t bytes, uint64_t stage_bytes, const char* prefix) {
    im.bytes = bytes;
    if (!prefix) {
        cudaError_t e = cudaMallocHost(&im.host, bytes);
        if (e != cudaSuccess) {
            im.host = nullptr;
            return ctx_fail(ctx, NSAT_ENOMEM, "pinned host image of " + std::to_string(bytes) + " bytes: " +
                                                  cudaGetErrorString(e));
        }
        return NSAT_OK;
    }
    const long long ns = (long long)std::chrono::duration_cast<std::chrono::nanoseconds>(
                             std::chrono::system_clock::now().time_since_epoch()).count();
    im.path = std::string(prefix) + "greedy_temp_" + std::to_string(ns);
    im.fd = open(im.path.c_str(), O_RDWR | O_CREAT | O_TRUNC, 0600);
    if (im.fd < 0) {
        const std::string p = im.path;
        im.path.clear();
        return ctx_fail(ctx, NSAT_EINVAL, "cannot create image file " + p);
    }
    if (ftruncate(im.fd, (off_t)bytes) != 0) return ctx_fail(ctx, NSAT_ENOMEM, "cannot size image file");
    GCK(cudaMallocHost(&im.stage, stage_bytes));
    im.stage_bytes = stage_bytes;
    return NSAT_OK;
}

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
    const uint64_t pbytes = packed_bytes(L, bits), cbytes = packed_bytes(chunk, bits);
    GCK(cudaSetDevice(ctx_device(ctx)));
    Image im;
    if (int rc = open_image(ctx, im, packed_bytes(1ull << n, bits), std::max(pbytes, cbytes), o->file_prefix))
        return rc;
    DevBufs d;
    GCK(cudaMalloc(&d.chunk, chunk * 8));
    GCK(cudaMalloc(&d.packed, std::max(pbytes, cbytes)));
    bool any_stop = false;
    if (int rc = build_image(ctx, c, im, d, lb, &any_stop, r)) return rc;
    cudaFree(d.chunk);
    d.chunk = nullptr;
    if (!any_stop) {
        r->wall_ms = now_ms() - t0;
        return NSAT_OK;
    }
    GCK(cudaMalloc(&d.dest, L * 8));
    GCK(cudaMalloc(&d.second, L * 8));
    GCK(cudaMalloc(&d.best, 8));
    cudaStream_t st = ctx_stream(ctx);
    const int sms = ctx_sm_count(ctx);
    cudaEvent_t e0, e1;
    GCK(cudaEventCreate(&e0));
    GCK(cudaEventCreate(&e1));
    struct EvGuard {
        cudaEvent_t a, b;
        ~EvGuard() { cudaEventDestroy(a); cudaEventDestroy(b); }
    } eg{e0, e1};
    for (uint32_t stage = 0; stage < n; stage++) {
        for (uint32_t i = 0; i < P; i++) {
            const uint64_t start_i = (uint64_t)i * L;
            if (int rc = image_to_device(ctx, im, (uint64_t)i * pbytes, pbytes, d.packed, st, r)) return rc;
            KCK(nsat_greedy_unpack(d.packed, L, bits, d.dest, sms, st));
            for (uint32_t j = 0; j < P; j++) {
                if (j != i) {
                    if (int rc = image_to_device(ctx, im, (uint64_t)j * pbytes, pbytes, d.packed, st, r)) return rc;
                    KCK(nsat_greedy_unpack(d.packed, L, bits, d.second, sms, st));
                } else {
                    GCK(cudaMemcpyAsync(d.second, d.dest, L * 8, cudaMemcpyDeviceToDevice, st));
                }
                GCK(cudaEventRecord(e0, st));
                KCK(nsat_greedy_join(d.dest, L, d.second, (uint64_t)j * L, L, n, sms, st));
                GCK(cudaEventRecord(e1, st));
                GCK(cudaEventSynchronize(e1));
                float ms = 0;
                GCK(cudaEventElapsedTime(&ms, e0, e1));
                r->join_ms += ms;
                r->joins++;
            }
            uint64_t best = ~0ull;
            GCK(cudaMemcpyAsync(d.best, &best, 8, cudaMemcpyHostToDevice, st));
            KCK(nsat_greedy_find(d.dest, start_i, L, n, o->unknowns, d.best, sms, st));
            GCK(cudaMemcpyAsync(&best, d.best, 8, cudaMemcpyDeviceToHost, st));
            GCK(cudaStreamSynchronize(st));
            if (best != ~0ull) {
                uint64_t e = 0;
                GCK(cudaMemcpy(&e, d.dest + (best - start_i), 8, cudaMemcpyDeviceToHost));
                r->found = 1;
                r->start = best;
                r->end = e & ((1ull << n) - 1);
                r->stage = stage;
                r->partition = i;
                r->wall_ms = now_ms() - t0;
                return NSAT_OK;
            }
            KCK(nsat_greedy_pack(d.dest, L, bits, d.packed, sms, st));
            if (int rc = device_to_image(ctx, im, (uint64_t)i * pbytes, pbytes, d.packed, st, r)) return rc;
            GCK(cudaStreamSynchronize(st));
        }
    }
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
    uint32_t pbits = 0;
    if (int rc = check_opts(ctx, n, &o, &pbits)) return rc;
    const uint64_t total = packed_bytes(1ull << n, bits);
    if (nwords * 8 < total) return ctx_fail(ctx, NSAT_EINVAL, "image buffer too small");
    const uint32_t lb = std::min(pbits + 2, n - 10);
    const uint64_t chunk = 1ull << (n - lb);
    const uint64_t cbytes = packed_bytes(chunk, bits);
    GCK(cudaSetDevice(ctx_device(ctx)));
    Image im;
    if (int rc = open_image(ctx, im, total, cbytes, file_prefix)) return rc;
    DevBufs d;
    GCK(cudaMalloc(&d.chunk, chunk * 8));
    GCK(cudaMalloc(&d.packed, cbytes));
    nsat_greedy_result r{};
    bool any = false;
    if (int rc = build_image(ctx, c, im, d, lb, &any, &r)) return rc;
    if (im.host) {
        memcpy(words, im.host, total);
    } else if (!pread_all(im.fd, words, total, 0)) {
        return ctx_fail(ctx, NSAT_EINVAL, "image file read failed");
    }
    return NSAT_OK;
}

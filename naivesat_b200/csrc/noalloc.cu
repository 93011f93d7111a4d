// noalloc.cu -- nsat_qsat_solve_noalloc: the QSAT solve without any device
// allocation, for callers that cannot call cudaMalloc.
//
// Who needs it: a host that runs the solver inside a serving process whose
// device memory is owned by another allocator (a caching allocator or a fixed
// per-tenant budget), or next to latency-critical streams.  cudaMalloc and
// cudaFree can synchronize the whole device and stall those streams, and a
// first-touch allocation can fail or breach the budget in the middle of a
// request.  nsat_qsat_solve allocates its last-CTA scratch lazily
// (cudaMalloc on first use and whenever a launch needs more); this variant
// uses the fixed area below instead.
#include <cuda_runtime.h>

#include <cstring>
#include <mutex>
#include <string>

#include "internal.h"
#include "nsat.h"

namespace {

// Scratch of the QSAT last-CTA tail: one byte per CTA plus a ping-pong half
// (2 << CB bytes per launch).  64 KiB covers launches of up to 2^15 CTAs.
// Every GPU that loads libnsat.so holds this array until the process exits.
constexpr size_t kScratchBytes = NSAT_NOALLOC_SCRATCH_BYTES;
static __device__ __align__(256) unsigned char g_noalloc_scratch[kScratchBytes];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
unsigned char* g_ptr[kMaxDevices] = {};

// Device address of g_noalloc_scratch on `device` (the name is only a host
// stand-in in host code).  Looked up once per device, with that device
// current; the first lookup may load this library's device module.
int scratch_on(int device, unsigned char** out) {
    if (device < 0 || device >= kMaxDevices) return NSAT_EINVAL;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_ptr[device]) {
        int prev = -1;
        cudaGetDevice(&prev);
        if (cudaSetDevice(device) != cudaSuccess) return NSAT_ECUDA;
        void* p = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (prev >= 0 && prev != device) cudaSetDevice(prev);
        if (e != cudaSuccess || !p) return NSAT_ECUDA;
        g_ptr[device] = static_cast<unsigned char*>(p);
    }
    *out = g_ptr[device];
    return NSAT_OK;
}

}  // namespace

extern "C" int nsat_qsat_solve_noalloc(nsat_ctx* ctx, nsat_circuit* c, const uint8_t* quants,
                                       const nsat_qsat_opts* opts, nsat_qsat_result* res) {
    if (!ctx || !c || !quants || !res) return NSAT_EINVAL;
    unsigned char* scratch = nullptr;
    int rc = scratch_on(nsat::ctx_device(ctx), &scratch);
    if (rc != NSAT_OK) return rc;
    // Nothing in the area has to start at zero: every launch writes each
    // byte it later reads (one per CTA, then the tail's ping-pong half).
    return nsat::qsat_solve_with_scratch(ctx, c, quants, opts, res, scratch, kScratchBytes);
}

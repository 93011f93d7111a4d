// static_kernels.cu -- circuit-independent sm_100a kernels, compiled by nvcc:
// the SATOSTOP pointer-doubling round (join_nexts + find_solution fused) and
// the LOP3 issue-rate probe.
#include <cuda_runtime.h>
#include <stdint.h>

#include "static_kernels.h"

typedef unsigned int u32;
typedef unsigned long long u64;

namespace {

// Entry formats of the next-state table.
//   FMT 0: u32  next | STOP << n            (n <= 31)
//   FMT 1: u64  next | STOP << n            (n <= 63)
//   FMT 2: u64  (next | STOP << n) | dist << 32   (n <= 31)
template <int FMT> struct EntryT { typedef u64 type; };
template <> struct EntryT<0> { typedef u32 type; };

template <int FMT, typename E>
__device__ __forceinline__ E combine(E v, E w) {
    if constexpr (FMT == 2) {
        return (w & 0xffffffffull) | (((v >> 32) + (w >> 32)) << 32);
    } else {
        (void)v;
        return w;
    }
}

__device__ __forceinline__ u64 warp_min(u64 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        u64 w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

// One synchronous doubling round (greedysatostop.rs:858-866 join_nexts, done
// out of place so that every entry advances exactly 2^r evaluations), fused
// with find_solution (greedysatostop.rs:883-895): the lowest start whose entry
// now has STOP is min-reduced into st->best[r].
template <int FMT>
__global__ void __launch_bounds__(256) join_round(const typename EntryT<FMT>::type* __restrict__ src,
                                                  typename EntryT<FMT>::type* __restrict__ dst,
                                                  u64 N, u32 n, u32 u, u32 r, u32 mode,
                                                  NsatJoinState* __restrict__ st) {
    typedef typename EntryT<FMT>::type E;
    if (r > 1) {
        const u64 pb = *(volatile u64*)&st->best[r - 1];
        if (pb != ~0ull && (mode == 0 || pb == 0)) {
            // solved in an earlier round: carry the answer forward, do no work
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                st->best[r] = pb;
                if (st->final_round == 0) st->final_round = r - 1;
            }
            return;
        }
    }
    const E stop = (E)1 << n;
    const E nmask = stop - 1;
    const u64 smask = (1ull << (n - u)) - 1ull;
    u64 best = ~0ull;
    const u64 S = (u64)gridDim.x * blockDim.x;
    const u64 t0 = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    // four independent gathers in flight per thread
    for (u64 i = t0; i < N; i += 4 * S) {
        E v[4];
        bool ok[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const u64 j = i + (u64)k * S;
            ok[k] = j < N;
            v[k] = ok[k] ? src[j] : stop;
        }
        E w[4];
#pragma unroll
        for (int k = 0; k < 4; k++) w[k] = (v[k] & stop) ? v[k] : src[(u64)(v[k] & nmask)];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const u64 j = i + (u64)k * S;
            if (!ok[k]) continue;
            const E o = (v[k] & stop) ? v[k] : combine<FMT>(v[k], w[k]);
            dst[j] = o;
            if ((j & smask) == 0 && (o & stop) && j < best) best = j;
        }
    }
    best = warp_min(best);
    if ((threadIdx.x & 31) == 0 && best != ~0ull) atomicMin(&st->best[r], best);
}

// Random-gather probe: 8-byte reads from a table of 2^logn entries at
// addresses spread by a multiplicative hash of the item index (every address
// is known up front, four loads in flight per thread), folded into one word
// per thread so no load is dropped.  Its rate is the ceiling of the joins'
// gathers, which no streaming-copy figure describes.
__global__ void __launch_bounds__(256) gather_probe(const u64* __restrict__ table, u32 logn, u64 items,
                                                    u64* __restrict__ out) {
    const u64 S = (u64)gridDim.x * blockDim.x;
    const u64 t0 = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    u64 acc = 0;
    for (u64 i = t0; i < items; i += 4 * S) {
        u64 v[4];
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const u64 j = i + (u64)k * S;
            const u64 h = (j * 0x9E3779B97F4A7C15ull) >> (64 - logn);
            v[k] = j < items ? __ldg(table + h) : 0;
        }
        acc ^= v[0] ^ v[1] ^ v[2] ^ v[3];
    }
    out[t0] = acc;
}

// LOP3 issue-rate probe: 8 independent chains per thread, each step mixes
// three previous values so no two steps fold into one LUT.
template <int LUT>
__device__ __forceinline__ u32 lop3(u32 a, u32 b, u32 c) {
    u32 d;
    asm volatile("lop3.b32 %0, %1, %2, %3, %4;" : "=r"(d) : "r"(a), "r"(b), "r"(c), "n"(LUT));
    return d;
}

__global__ void __launch_bounds__(256) lop3_probe(u32* out, int iters, u64* clk) {
    u32 a0 = threadIdx.x * 0x9e3779b9u + blockIdx.x, a1 = a0 ^ 0x85ebca6bu, a2 = a0 * 3u + 7u,
        a3 = a0 ^ 0xc2b2ae35u, a4 = a1 + a2, a5 = a2 ^ a3, a6 = a0 + 0x27d4eb2fu, a7 = a3 * 5u;
    u64 c0 = clock64();
    for (int i = 0; i < iters; i++) {
        u32 b0 = lop3<0x96>(a0, a1, a2), b1 = lop3<0xe8>(a1, a2, a3), b2 = lop3<0x1e>(a2, a3, a4),
            b3 = lop3<0x78>(a3, a4, a5), b4 = lop3<0x96>(a4, a5, a6), b5 = lop3<0xe8>(a5, a6, a7),
            b6 = lop3<0x1e>(a6, a7, a0), b7 = lop3<0x78>(a7, a0, a1);
        a0 = lop3<0x96>(b0, b1, b2); a1 = lop3<0xe8>(b1, b2, b3); a2 = lop3<0x1e>(b2, b3, b4);
        a3 = lop3<0x78>(b3, b4, b5); a4 = lop3<0x96>(b4, b5, b6); a5 = lop3<0xe8>(b5, b6, b7);
        a6 = lop3<0x1e>(b6, b7, b0); a7 = lop3<0x78>(b7, b0, b1);
    }
    u64 c1 = clock64();
    u32 r = a0 ^ a1 ^ a2 ^ a3 ^ a4 ^ a5 ^ a6 ^ a7;
    if (r == 0x12345678u) out[blockIdx.x * blockDim.x + threadIdx.x] = r;   // keeps the chains live
    if (threadIdx.x == 0) {
        u32 smid;
        asm volatile("mov.u32 %0, %%smid;" : "=r"(smid));
        clk[3 * blockIdx.x] = c0;
        clk[3 * blockIdx.x + 1] = c1;
        clk[3 * blockIdx.x + 2] = smid;
    }
}

}  // namespace

extern "C" int nsat_launch_join_round(int fmt, const void* src, void* dst, uint64_t N, uint32_t n,
                                      uint32_t u, uint32_t r, uint32_t mode, NsatJoinState* st,
                                      int sm_count, cudaStream_t stream) {
    const unsigned threads = 256;
    u64 want = (N + 4ull * threads - 1) / (4ull * threads);
    u64 cap = (u64)sm_count * 8ull;
    unsigned blocks = (unsigned)(want < cap ? want : cap);
    if (blocks == 0) blocks = 1;
    switch (fmt) {
    case 0:
        join_round<0><<<blocks, threads, 0, stream>>>((const u32*)src, (u32*)dst, N, n, u, r, mode, st);
        break;
    case 1:
        join_round<1><<<blocks, threads, 0, stream>>>((const u64*)src, (u64*)dst, N, n, u, r, mode, st);
        break;
    case 2:
        join_round<2><<<blocks, threads, 0, stream>>>((const u64*)src, (u64*)dst, N, n, u, r, mode, st);
        break;
    default:
        return -1;
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

extern "C" int nsat_launch_gather_probe(const uint64_t* table, uint32_t logn, uint64_t items, uint64_t* out,
                                        int blocks, cudaStream_t stream) {
    gather_probe<<<blocks, 256, 0, stream>>>((const u64*)table, logn, items, (u64*)out);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

extern "C" int nsat_launch_lop3_probe(uint32_t* out, int blocks, int iters, uint64_t* clk,
                                      cudaStream_t stream) {
    lop3_probe<<<blocks, 256, 0, stream>>>(out, iters, (u64*)clk);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

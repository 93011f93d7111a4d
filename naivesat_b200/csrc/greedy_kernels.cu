// greedy_kernels.cu -- device side of the partitioned greedysatostop solver
// (greedysatostop -p): the packed table image and the partition joins.
//
// Image layout (greedysatostop.rs MemImage, 308-489): entry i of a state
// space of n bits is n+1 bits (next | STOP << n) at bit i*(n+1) of a
// little-endian u64 array; an entry may straddle two words.  Partitions hold
// multiples of 64 entries, so every partition starts on a word boundary.
// The partition being updated is unpacked to u64 entries (an in-place join
// on packed entries would race: entries share words); the partitions it
// gathers from are read packed.
#include <cuda_runtime.h>
#include <stdint.h>

#include "greedy_kernels.h"

typedef unsigned long long u64;
typedef unsigned int u32;

namespace {

__global__ void unpack_kernel(const u64* __restrict__ packed, u64 count, u32 bits, u64* __restrict__ out) {
    const u64 mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const u64 b = i * bits;
        const u64 w = b >> 6;
        const u32 o = (u32)(b & 63);
        u64 v = packed[w] >> o;
        if (o + bits > 64) v |= packed[w + 1] << (64 - o);
        out[i] = v & mask;
    }
}

// One output word per thread: the bits of every entry that overlaps it.
__global__ void pack_kernel(const u64* __restrict__ in, u64 nwords, u32 bits, u64* __restrict__ packed) {
    const u64 mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 w = (u64)blockIdx.x * blockDim.x + threadIdx.x; w < nwords; w += stride) {
        const u64 lo = w << 6;
        const u64 first = lo / bits, last = (lo + 63) / bits;
        u64 acc = 0;
        for (u64 e = first; e <= last; e++) {
            const u64 v = in[e] & mask;
            const u64 eb = e * bits;
            if (eb >= lo) acc |= v << (u32)(eb - lo);      // eb - lo < 64 because e <= last
            else acc |= v >> (u32)(lo - eb);               // lo - eb < bits <= 64
        }
        packed[w] = acc;
    }
}

// greedysatostop.rs MemImage::join_nexts (433-481): an entry that has not
// stopped and whose next state lies in `second` takes second's entry.
__global__ void join_kernel(u64* __restrict__ dest, u64 count, const u64* __restrict__ second, u64 start2,
                            u64 count2, u32 n) {
    const u64 state_mask = (1ull << n) - 1;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const u64 v = dest[i];
        if ((v >> n) & 1ull) continue;
        const u64 off = (v & state_mask) - start2;     // wraps above count2 when next < start2
        if (off < count2) dest[i] = __ldg(second + off);
    }
}

// The same join with `second` still packed (bits = n+1 per entry): the
// gather reads the one or two words that hold the entry.
__global__ void join_packed_kernel(u64* __restrict__ dest, u64 count, const u64* __restrict__ second, u64 start2,
                                   u64 count2, u32 n) {
    const u32 bits = n + 1;
    const u64 state_mask = (1ull << n) - 1;
    const u64 mask = bits >= 64 ? ~0ull : ((1ull << bits) - 1);
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += stride) {
        const u64 v = dest[i];
        if ((v >> n) & 1ull) continue;
        const u64 off = (v & state_mask) - start2;
        if (off >= count2) continue;
        const u64 b = off * bits;
        const u64 w = b >> 6;
        const u32 o = (u32)(b & 63);
        u64 x = __ldg(second + w) >> o;
        if (o + bits > 64) x |= __ldg(second + w + 1) << (64 - o);
        dest[i] = x & mask;
    }
}

// greedysatostop.rs MemImage::find_solution (482-507): the lowest unknown
// start of the partition (low n-u bits zero) whose entry has STOP.
__global__ void find_kernel(const u64* __restrict__ dest, u64 start, u64 count, u32 n, u32 unknowns,
                            u64* __restrict__ best) {
    const u64 before = (n - unknowns) >= 64 ? ~0ull : ((1ull << (n - unknowns)) - 1);
    const u64 step = before + 1;
    const u64 us0 = (start & before) ? (start & ~before) + step : (start & ~before);
    const u64 end = start + count;
    if (us0 >= end) return;
    const u64 cands = (end - us0 + step - 1) / step;
    const u64 stride = (u64)gridDim.x * blockDim.x;
    for (u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x; k < cands; k += stride) {
        const u64 s = us0 + k * step;
        if ((dest[s - start] >> n) & 1ull) atomicMin(best, s);
    }
}

unsigned grid_for(u64 items, int sms) {
    const u64 want = (items + 255) / 256;
    const u64 cap = (u64)sms * 8;
    return (unsigned)(want < 1 ? 1 : (want > cap ? cap : want));
}

}  // namespace

extern "C" int nsat_greedy_unpack(const uint64_t* packed, uint64_t count, uint32_t bits, uint64_t* out, int sms,
                                  cudaStream_t st) {
    unpack_kernel<<<grid_for(count, sms), 256, 0, st>>>((const u64*)packed, count, bits, (u64*)out);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

extern "C" int nsat_greedy_pack(const uint64_t* in, uint64_t count, uint32_t bits, uint64_t* packed, int sms,
                                cudaStream_t st) {
    const u64 nwords = (count * bits) >> 6;   // count is a multiple of 64
    pack_kernel<<<grid_for(nwords, sms), 256, 0, st>>>((const u64*)in, nwords, bits, (u64*)packed);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

extern "C" int nsat_greedy_join(uint64_t* dest, uint64_t count, const uint64_t* second, uint64_t start2,
                                uint64_t count2, uint32_t n, int sms, cudaStream_t st) {
    join_kernel<<<grid_for(count, sms), 256, 0, st>>>((u64*)dest, count, (const u64*)second, start2, count2, n);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

extern "C" int nsat_greedy_join_packed(uint64_t* dest, uint64_t count, const uint64_t* second_packed, uint64_t start2,
                                       uint64_t count2, uint32_t n, int sms, cudaStream_t st) {
    join_packed_kernel<<<grid_for(count, sms), 256, 0, st>>>((u64*)dest, count, (const u64*)second_packed, start2,
                                                             count2, n);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

extern "C" int nsat_greedy_find(const uint64_t* dest, uint64_t start, uint64_t count, uint32_t n, uint32_t unknowns,
                                uint64_t* best, int sms, cudaStream_t st) {
    find_kernel<<<grid_for(count, sms), 256, 0, st>>>((const u64*)dest, start, count, n, unknowns, (u64*)best);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

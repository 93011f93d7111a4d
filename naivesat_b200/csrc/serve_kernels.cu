// serve_kernels.cu -- the batched serving engine's kernel: a LOP3 bytecode
// interpreter that evaluates many different circuits in one launch.
//
// Per-request NVRTC compilation costs 0.1-1.5 s per circuit, far more than
// the device work of most serving requests, so serving does not specialise
// kernels: every job is a program of 3-input LUT instructions over "slots"
// (the LUT cover of its circuit, slot-allocated by liveness).  Each warp
// evaluates 32 words (1024 assignments) per iteration and 32 iterations per
// tile (2^15 assignments); slot values live in shared memory laid out
// [slot][lane] (conflict-free), each instruction is applied with a runtime
// truth table through a 7-LOP3 mux tree over warp-uniform masks.
//
// Scheduling is on the device: every warp starts at its own job of the epoch
// table and claims tiles of that job's slice with an atomic cursor, moving on
// round-robin when a slice is used up; a warp ends after one full pass finds
// nothing left (no waiting on anything).
#include <cuda_runtime.h>
#include <stdint.h>

#include "serve_common.h"
#include "serve_kernels.h"

typedef unsigned int u32;
typedef unsigned long long u64;

namespace {

template <int LUT>
__device__ __forceinline__ u32 lop3(u32 a, u32 b, u32 c) {
    u32 d;
    asm("lop3.b32 %0, %1, %2, %3, %4;" : "=r"(d) : "r"(a), "r"(b), "r"(c), "n"(LUT));
    return d;
}

// s ? x1 : x0, bitwise
__device__ __forceinline__ u32 mux(u32 s, u32 x1, u32 x0) { return lop3<0xCA>(s, x1, x0); }

// 3-input LUT with a runtime truth table (row = a<<2 | b<<1 | c)
__device__ __forceinline__ u32 lut3(u32 a, u32 b, u32 c, u32 tt) {
    const u32 t0 = 0u - (tt & 1u), t1 = 0u - ((tt >> 1) & 1u), t2 = 0u - ((tt >> 2) & 1u),
              t3 = 0u - ((tt >> 3) & 1u), t4 = 0u - ((tt >> 4) & 1u), t5 = 0u - ((tt >> 5) & 1u),
              t6 = 0u - ((tt >> 6) & 1u), t7 = 0u - ((tt >> 7) & 1u);
    const u32 x01 = mux(c, t1, t0), x23 = mux(c, t3, t2), x45 = mux(c, t5, t4), x67 = mux(c, t7, t6);
    return mux(a, mux(b, x67, x45), mux(b, x23, x01));
}

__device__ __forceinline__ u64 warp_min(u64 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        u64 w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

__device__ __forceinline__ u32 tree_rt(u32 y, u64 allbits, int lvl, int cnt) {
    for (int j = 0; j < cnt; j++) {
        if ((allbits >> (lvl + j)) & 1ull) y &= (y >> (1 << j));
        else y |= (y >> (1 << j));
    }
    return y;
}

__device__ __forceinline__ u32 unit_mask(int k) {
    return k == 0 ? 0xffffffffu : k == 1 ? 0x55555555u : k == 2 ? 0x11111111u
         : k == 3 ? 0x01010101u : k == 4 ? 0x00010001u : 0x1u;
}

__device__ __forceinline__ void transpose32(u32* a) {
#pragma unroll
    for (int j = 16; j > 0; j >>= 1) {
        const u32 m = j == 16 ? 0x0000ffffu : j == 8 ? 0x00ff00ffu : j == 4 ? 0x0f0f0f0fu
                    : j == 2 ? 0x33333333u : 0x55555555u;
#pragma unroll
        for (int k = 0; k < 32; k++) {
            if ((k & j) == 0) {
                const u32 t = ((a[k] >> j) ^ a[k + j]) & m;
                a[k + j] ^= t;
                a[k] ^= t << j;
            }
        }
    }
}

// Runs a job's program on one word per lane; slots S[slot * 32 + lane].
__device__ __forceinline__ void run_program(const srv_u64* __restrict__ prog, u32 ninstr,
                                            u32* __restrict__ S, u32 lane) {
    u32 i = 0;
    for (; i + 2 <= ninstr; i += 2) {
        const u64 p0 = __ldg(prog + i), p1 = __ldg(prog + i + 1);
        const u32 a0 = S[((u32)p0 & 0xfffu) * 32 + lane], b0 = S[((u32)(p0 >> 12) & 0xfffu) * 32 + lane],
                  c0 = S[((u32)(p0 >> 24) & 0xfffu) * 32 + lane];
        S[((u32)(p0 >> 36) & 0xfffu) * 32 + lane] = lut3(a0, b0, c0, (u32)(p0 >> 48) & 0xffu);
        const u32 a1 = S[((u32)p1 & 0xfffu) * 32 + lane], b1 = S[((u32)(p1 >> 12) & 0xfffu) * 32 + lane],
                  c1 = S[((u32)(p1 >> 24) & 0xfffu) * 32 + lane];
        S[((u32)(p1 >> 36) & 0xfffu) * 32 + lane] = lut3(a1, b1, c1, (u32)(p1 >> 48) & 0xffu);
    }
    if (i < ninstr) {
        const u64 p0 = __ldg(prog + i);
        const u32 a0 = S[((u32)p0 & 0xfffu) * 32 + lane], b0 = S[((u32)(p0 >> 12) & 0xfffu) * 32 + lane],
                  c0 = S[((u32)(p0 >> 24) & 0xfffu) * 32 + lane];
        S[((u32)(p0 >> 36) & 0xfffu) * 32 + lane] = lut3(a0, b0, c0, (u32)(p0 >> 48) & 0xffu);
    }
}

__device__ __forceinline__ u32 read_out(const u32* S, const uint16_t* outs, u32 j, u32 lane) {
    const uint16_t o = __ldg(outs + j);
    const u32 v = S[(o & 0x7fffu) * 32 + lane];
    return (o & 0x8000u) ? ~v : v;
}

// Evaluates tile `tile` of job `J` with this warp.
__device__ void do_tile(SrvJob* J, u64 tile, u32* __restrict__ S, u32 lane, uint8_t* __restrict__ vals) {
    const u32 nb = J->nb;
    const u64 tile_base = tile << SRV_TILE_BITS;     // first assignment of the tile
    // inputs fixed for the tile: word lanes, warp lanes, tile bits
    for (u32 p = 0; p < nb && p < SRV_MAX_NB; p++) {
        const int s = J->in_slot[p];
        if (s < 0 || (p >= 10 && p < 15)) continue;
        u32 v;
        if (p < 5) v = p == 0 ? 0xAAAAAAAAu : p == 1 ? 0xCCCCCCCCu : p == 2 ? 0xF0F0F0F0u : p == 3 ? 0xFF00FF00u : 0xFFFF0000u;
        else if (p < 10) v = 0u - ((lane >> (p - 5)) & 1u);
        else v = 0u - (u32)((tile_base >> p) & 1ull);
        S[s * 32 + lane] = v;
    }
    __syncwarp();
    const u32 kind = J->kind;
    u32 cnt = 0, first_it = 0xffffffffu, first_bit = 0;
    u64 cand = ~0ull;
    u32 acc = 0;
    const u32 M = J->m;
    const u64 allbits = J->allbits;
    const u32 dec_all = J->q0all;
    for (u32 it = 0; it < 32; it++) {
        for (u32 p = 10; p < 15 && p < nb; p++) {
            const int s = J->in_slot[p];
            if (s >= 0) S[s * 32 + lane] = 0u - ((it >> (p - 10)) & 1u);
        }
        __syncwarp();
        run_program(J->prog, J->ninstr, S, lane);
        __syncwarp();
        if (kind == SRV_SAT) {
            const u32 y = read_out(S, J->outs, 0, lane);
            cnt += __popc(y);
            if (y != 0u && first_it == 0xffffffffu) { first_it = it; first_bit = __ffs(y) - 1; }
        } else if (kind == SRV_QSAT) {
            u32 y = read_out(S, J->outs, 0, lane);
            const u64 wbase = tile_base + ((u64)it << 10);      // first item of this warp iteration
            if (M < 5) {
                y = tree_rt(y, allbits, 0, (int)M);
                const u32 d = (dec_all ? ~y : y) & unit_mask((int)M);
                if (d != 0u && cand == ~0ull) cand = ((wbase + ((u64)lane << 5)) >> M) + ((__ffs(d) - 1) >> M);
                continue;
            }
            y = tree_rt(y, allbits, 0, 5);
            u32 b = __ballot_sync(0xffffffffu, y & 1u);
            if (M < 10) {
                b = tree_rt(b, allbits, 5, (int)M - 5);
                const u32 d = (dec_all ? ~b : b) & unit_mask((int)M - 5);
                if (d != 0u && cand == ~0ull) cand = (wbase >> M) + ((__ffs(d) - 1) >> (M - 5));
                continue;
            }
            b = tree_rt(b, allbits, 5, 5);
            acc |= (b & 1u) << it;
        } else {   // SRV_TABLE
            u32 o[32];
#pragma unroll
            for (int k = 0; k < 32; k++) o[k] = (u32)k < J->nout ? read_out(S, J->outs, k, lane) : 0u;
            transpose32(o);
            const u64 w = (tile_base >> 5) + ((u64)it << 5) + lane;   // word index
            const u32 lanes = J->n >= 5 ? 32u : (1u << J->n);
            const u64 states = 1ull << J->n;
            if ((w << 5) < states) {
                u64* dst = J->table + (w << 5);
                for (u32 l = 0; l < lanes; l++) dst[l] = (u64)o[l] | (1ull << 32);
            }
            const u32 stop = read_out(S, J->outs, J->nout - 1, lane);
            if (__any_sync(0xffffffffu, stop != 0u) && lane == 0) atomicOr(&J->any, 1u);
        }
    }
    if (kind == SRV_SAT) {
        u64 idx = ~0ull;
        if (first_it != 0xffffffffu) idx = tile_base + ((u64)first_it << 10) + ((u64)lane << 5) + first_bit;
        idx = warp_min(idx);
        cnt = __reduce_add_sync(0xffffffffu, cnt);
        if (lane == 0 && cnt) {
            atomicAdd(&J->count, (u64)cnt);
            atomicMin(&J->min_idx, idx);
        }
    } else if (kind == SRV_QSAT) {
        if (M < 10) {
            cand = warp_min(cand);
            if (lane == 0 && cand != ~0ull) atomicMin(&J->min_idx, cand);
        } else if (M < SRV_TILE_BITS) {
            const u32 y = tree_rt(acc, allbits, 10, (int)M - 10);
            const u32 d = (dec_all ? ~y : y) & unit_mask((int)M - 10);
            if (lane == 0 && d != 0u) atomicMin(&J->min_idx, (tile_base >> M) + ((__ffs(d) - 1) >> (M - 10)));
        } else {
            const u32 y = tree_rt(acc, allbits, 10, 5);
            if (lane == 0) vals[J->val_off + (tile - J->tile_begin)] = (uint8_t)(y & 1u);
        }
    }
    __syncwarp();
}

__global__ void __launch_bounds__(SRV_WARPS_PER_CTA * 32) serve_epoch(const SrvEpoch* __restrict__ hdr, SrvJob* __restrict__ jobs,
                                                   u32 max_slots, uint8_t* __restrict__ vals) {
    extern __shared__ u32 smem[];
    const u32 njobs = hdr->njobs;
    const u32 lane = threadIdx.x & 31u;
    const u32 wid = threadIdx.x >> 5;
    u32* S = smem + (size_t)wid * max_slots * 32;
    const u32 gw = blockIdx.x * (blockDim.x >> 5) + wid;
    u32 j = njobs ? gw % njobs : 0;
    u32 dry = 0;     // consecutive jobs found exhausted
    while (dry < njobs) {
        SrvJob* J = jobs + j;
        u64 tile = 0;
        if (lane == 0) tile = atomicAdd(&J->claim, 1ull);
        tile = __shfl_sync(0xffffffffu, tile, 0);
        if (tile >= J->tile_end) {
            dry++;
            j = (j + 1 == njobs) ? 0 : j + 1;
            continue;
        }
        dry = 0;
        do_tile(J, tile, S, lane, vals);
    }
}

}  // namespace

extern "C" int nsat_launch_serve_epoch(const SrvEpoch* hdr, SrvJob* jobs, uint32_t max_slots, uint8_t* vals,
                                       int grid, cudaStream_t stream) {
    // the dynamic shared memory limit was raised by nsat_serve_occupancy
    const size_t smem = (size_t)SRV_WARPS_PER_CTA * max_slots * 32 * sizeof(u32);
    serve_epoch<<<grid, SRV_WARPS_PER_CTA * 32, smem, stream>>>(hdr, jobs, max_slots, vals);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

extern "C" int nsat_serve_occupancy(uint32_t max_slots, int* ctas_per_sm) {
    const size_t smem = (size_t)SRV_WARPS_PER_CTA * max_slots * 32 * sizeof(u32);
    if (cudaFuncSetAttribute(serve_epoch, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem) != cudaSuccess)
        return -4;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, serve_epoch, SRV_WARPS_PER_CTA * 32, smem) ==
                   cudaSuccess ? 0 : -4;
}

// serve_kernels.cu -- the batched serving engine's kernel: a LOP3 bytecode
// interpreter that evaluates many different circuits in one launch.
//
// Per-request NVRTC compilation costs 0.06-0.7 s per circuit, far more than
// the device work of most serving requests, so serving does not specialise
// kernels: every job is a program of 3-input LUT instructions over "slots"
// (the LUT cover of its circuit, scheduled into groups of independent
// instructions and slot-allocated by liveness).  A CTA is one warp; each lane
// evaluates W words per program pass, and slot values live in the warp's
// shared memory laid out [slot][lane][word] (conflict-free vector accesses).
//
// The kernel is instantiated for each shape of serve_common.h (W words per
// lane, groups of G instructions, LUT evaluation by mux tree or by jump):
// - mux tree: a LUT with a run-time truth table is 7 lop3 over eight masks
//   that 8 byte permutes expand from the 16-byte record (W = 4: 28 lop3 and
//   8 prmt per instruction and warp);
// - jump: every lane of a warp runs the same program, so the truth table is
//   warp-uniform; a switch over its 256 values jumps to one lop3 per word
//   with the table as its immediate (W lop3 per instruction).
// Either way an instruction reads three slots and writes one: 16 bytes of
// shared-memory traffic per LUT-word, which bounds the interpreter at
// 128 B/clk/SM / 16 B = 8 LUT-words per SM clock.
// The slot decode is done with multiply-adds so that it runs on the FMA pipe.
// A group of G independent instructions keeps 3 * G shared loads in flight,
// and the records of the next group are loaded while the current one
// computes.
//
// Scheduling is on the device: every warp starts at its own job of the epoch
// table and claims tiles from the job's persistent cursor, moving on
// round-robin when the job's slice is used up.  The search for the next job
// with tiles left checks 32 jobs at a time, one per lane.  When no slice has
// planned tiles left, warps go on into the next quarter slice of SAT and
// SATOSTOP jobs that are not decided yet, and end when none has tiles left
// either (no waiting on anything).
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

template <int W>
struct Vals {
    u32 v[W];
};

template <int W>
__device__ __forceinline__ Vals<W> lds(const char* p) {
    Vals<W> r;
    if constexpr (W == 4) {
        const uint4 t = *reinterpret_cast<const uint4*>(p);
        r.v[0] = t.x; r.v[1] = t.y; r.v[2] = t.z; r.v[3] = t.w;
    } else {
        const uint2 t = *reinterpret_cast<const uint2*>(p);
        r.v[0] = t.x; r.v[1] = t.y;
    }
    return r;
}

template <int W>
__device__ __forceinline__ void sts(char* p, const Vals<W>& x) {
    if constexpr (W == 4) *reinterpret_cast<uint4*>(p) = make_uint4(x.v[0], x.v[1], x.v[2], x.v[3]);
    else *reinterpret_cast<uint2*>(p) = make_uint2(x.v[0], x.v[1]);
}

// Mask k of a spread truth table: byte k of {thi, tlo} with its sign bit
// replicated over all 32 bits (prmt in its default mode: a selector nibble
// with bit 3 set replicates the sign of the byte its low 3 bits select; the
// __byte_perm intrinsic is only defined for the low 3 bits).
template <int K>
__device__ __forceinline__ u32 tt_mask(u32 tlo, u32 thi) {
    u32 d;
    asm("prmt.b32 %0, %1, %2, %3;" : "=r"(d) : "r"(tlo), "r"(thi), "n"((8 | K) * 0x1111));
    return d;
}

struct Lut {
    u32 m0, m1, m2, m3, m4, m5, m6, m7;
};

__device__ __forceinline__ Lut expand(const uint4& r) {
    Lut t;
    t.m0 = tt_mask<0>(r.z, r.w); t.m1 = tt_mask<1>(r.z, r.w); t.m2 = tt_mask<2>(r.z, r.w); t.m3 = tt_mask<3>(r.z, r.w);
    t.m4 = tt_mask<4>(r.z, r.w); t.m5 = tt_mask<5>(r.z, r.w); t.m6 = tt_mask<6>(r.z, r.w); t.m7 = tt_mask<7>(r.z, r.w);
    return t;
}

// LUT through a mux tree over the truth-table masks (7 lop3)
__device__ __forceinline__ u32 lut_mux(u32 a, u32 b, u32 c, const Lut& t) {
    const u32 x01 = mux(c, t.m1, t.m0), x23 = mux(c, t.m3, t.m2), x45 = mux(c, t.m5, t.m4), x67 = mux(c, t.m7, t.m6);
    return mux(a, mux(b, x67, x45), mux(b, x23, x01));
}

// The truth table of a record as an 8-bit number: bit k of tt is the sign
// bit of byte k of {thi, tlo}.  (x >> 7) has those bits at 0, 8, 16, 24, and
// the product with 0x01020408 gathers them into bits 24..27 (every other
// partial product lands below bit 24 at a distinct position, or above bit
// 31), so the gather is two shifts and a multiply per word.
__device__ __forceinline__ u32 tt_of(u32 tlo, u32 thi) {
    const u32 lo = ((tlo >> 7) * 0x01020408u) >> 24;
    const u32 hi = ((thi >> 7) * 0x01020408u) >> 24;
    return lo | (hi << 4);
}

// One LUT on W words with its truth table as the lop3 immediate: the table
// is the same for the whole warp (every lane runs the same program), so the
// switch is a uniform jump and each word costs one lop3.
template <int T, int W>
__device__ __forceinline__ void lut_imm(const Vals<W>& a, const Vals<W>& b, const Vals<W>& c, Vals<W>& d) {
#pragma unroll
    for (int w = 0; w < W; w++) d.v[w] = lop3<T>(a.v[w], b.v[w], c.v[w]);
}

#define SRV_CASE(t) \
    case (t): lut_imm<(t), W>(a, b, c, d); break;
#define SRV_CASE4(t) SRV_CASE(t) SRV_CASE((t) + 1) SRV_CASE((t) + 2) SRV_CASE((t) + 3)
#define SRV_CASE16(t) SRV_CASE4(t) SRV_CASE4((t) + 4) SRV_CASE4((t) + 8) SRV_CASE4((t) + 12)
#define SRV_CASE64(t) SRV_CASE16(t) SRV_CASE16((t) + 16) SRV_CASE16((t) + 32) SRV_CASE16((t) + 48)

template <int W>
__device__ __forceinline__ Vals<W> lut_switch(u32 tt, const Vals<W>& a, const Vals<W>& b, const Vals<W>& c) {
    Vals<W> d;
    switch (tt & 255u) {
        SRV_CASE64(0)
        SRV_CASE64(64)
        SRV_CASE64(128)
        SRV_CASE64(192)
    }
    return d;
}

// Slot fields decoded with multiply-adds (FMA pipe) instead of masks and
// shifts (ALU pipe, the kernel's bound): hi = x * km >> 32 with km = 65536,
// lo = x - hi * km, byte offset = field * sb; km and sb come from the epoch
// header so they are not folded back into shifts.
struct Dec { u32 km, sb; };
__device__ __forceinline__ void fields(u32 x, const Dec& dc, u32* lo, u32* hi) {
    *hi = __umulhi(x, dc.km);
    *lo = x - *hi * dc.km;
}

// Runs a job's program once on this lane's W words.  Sl is the warp's slot
// area plus lane * W * 4.
template <int W, int G, bool DISPATCH>
__device__ __forceinline__ void run_program(const SrvIns* __restrict__ prog, u32 ngroups, char* __restrict__ Sl,
                                            const Dec& dc) {
    if (ngroups == 0) return;
    const uint4* P = reinterpret_cast<const uint4*>(prog);
    uint4 cur[G];
#pragma unroll
    for (int k = 0; k < G; k++) cur[k] = __ldg(P + k);
    for (u32 g = 0; g < ngroups; g++) {
        Vals<W> a[G], b[G], c[G];
        u32 dof[G];
#pragma unroll
        for (int k = 0; k < G; k++) {
            u32 al, ah, cl, ch;
            fields(cur[k].x, dc, &al, &ah);
            fields(cur[k].y, dc, &cl, &ch);
            a[k] = lds<W>(Sl + al * dc.sb);
            b[k] = lds<W>(Sl + ah * dc.sb);
            c[k] = lds<W>(Sl + cl * dc.sb);
            dof[k] = ch * dc.sb;
        }
        const uint4* nx = P + (size_t)(g + 1 < ngroups ? g + 1 : g) * G;
        uint4 nxt[G];
#pragma unroll
        for (int k = 0; k < G; k++) nxt[k] = __ldg(nx + k);
#pragma unroll
        for (int k = 0; k < G; k++) {
            Vals<W> d;
            if constexpr (DISPATCH) {
                d = lut_switch<W>(tt_of(cur[k].z, cur[k].w), a[k], b[k], c[k]);
            } else {
                const Lut t = expand(cur[k]);
#pragma unroll
                for (int w = 0; w < W; w++) d.v[w] = lut_mux(a[k].v[w], b[k].v[w], c[k].v[w], t);
            }
            sts<W>(Sl + dof[k], d);
        }
#pragma unroll
        for (int k = 0; k < G; k++) cur[k] = nxt[k];
    }
}

template <int W>
__device__ __forceinline__ Vals<W> read_out(const char* Sl, const uint16_t* outs, u32 j) {
    const uint16_t o = __ldg(outs + j);
    Vals<W> v = lds<W>(Sl + (u32)(o & 0x7fffu) * (32u * W * 4u));
    if (o & 0x8000u) {
#pragma unroll
        for (int w = 0; w < W; w++) v.v[w] = ~v.v[w];
    }
    return v;
}

// Enumeration inside a tile: bits 0-4 the bit of a word, 5-9 the lane,
// 10 .. 10+LOGW-1 which of the lane's words, the rest up to bit 14 the pass;
// bits from SRV_TILE_BITS up are the tile index.  Input slots are rewritten
// every pass because the program reuses slots of inputs it has finished
// reading.
template <int W>
__device__ __forceinline__ void set_inputs(const SrvJob* J, u64 tile_base, u32 it, u32 lane, char* Sl) {
    constexpr int LOGW = W == 4 ? 2 : 1;
    const u32 nb = J->nb < SRV_MAX_NB ? J->nb : SRV_MAX_NB;
    for (u32 p = 0; p < nb; p++) {
        const int s = J->in_slot[p];
        if (s < 0) continue;
        Vals<W> v;
#pragma unroll
        for (int w = 0; w < W; w++) {
            u32 x;
            if (p < 5) x = p == 0 ? 0xAAAAAAAAu : p == 1 ? 0xCCCCCCCCu : p == 2 ? 0xF0F0F0F0u : p == 3 ? 0xFF00FF00u : 0xFFFF0000u;
            else if (p < 10) x = 0u - ((lane >> (p - 5)) & 1u);
            else if (p < 10 + LOGW) x = 0u - (((u32)w >> (p - 10)) & 1u);
            else if (p < SRV_TILE_BITS) x = 0u - ((it >> (p - 10 - LOGW)) & 1u);
            else x = 0u - (u32)((tile_base >> p) & 1ull);
            v.v[w] = x;
        }
        sts<W>(Sl + (u32)s * (32u * W * 4u), v);
    }
}

// Evaluates tile `tile` of job `J` with this warp.
template <int W, int G, bool DISPATCH>
__device__ __forceinline__ void do_tile(SrvJob* J, u64 tile, char* __restrict__ Sl, u32 lane, uint8_t* __restrict__ vals,
                                        const Dec& dc) {
    constexpr u32 ITERS = 32u / W;                 // program passes per tile
    const u64 tile_base = tile << SRV_TILE_BITS;     // first assignment of the tile
    const u32 kind = J->kind;
    const SrvIns* prog = J->prog;
    const u32 ngroups = J->ngroups;
    u32 cnt = 0, first = 0xffffffffu;   // SAT: first (row, bit) with a solution, row = it * W + word
    u64 cand = ~0ull;
    u32 acc = 0;
    const u32 M = J->m;
    const u64 allbits = J->allbits;
    const u32 dec_all = J->q0all;
    for (u32 it = 0; it < ITERS; it++) {
        set_inputs<W>(J, tile_base, it, lane, Sl);
        run_program<W, G, DISPATCH>(prog, ngroups, Sl, dc);
        if (kind == SRV_SAT) {
            const Vals<W> y = read_out<W>(Sl, J->outs, 0);
#pragma unroll
            for (int w = 0; w < W; w++) {
                cnt += __popc(y.v[w]);
                if (first == 0xffffffffu && y.v[w]) first = ((it * W + w) << 5) | (u32)(__ffs(y.v[w]) - 1);
            }
        } else if (kind == SRV_QSAT) {
            const Vals<W> yy = read_out<W>(Sl, J->outs, 0);
#pragma unroll
            for (int w = 0; w < W; w++) {
                u32 y = yy.v[w];
                const u32 row = it * W + w;
                const u64 wbase = tile_base + ((u64)row << 10);   // first item of this word row
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
                acc |= (b & 1u) << row;
            }
        } else {   // SRV_TABLE
            const u32 lanes = J->n >= 5 ? 32u : (1u << J->n);
            const u64 states = 1ull << J->n;
            const u32 nout = J->nout;
            u32 stop_any = 0;
            for (int w = 0; w < W; w++) {
                u32 o[32];
#pragma unroll
                for (int k = 0; k < 32; k++) {
                    if ((u32)k < nout) o[k] = read_out<W>(Sl, J->outs, k).v[w];
                    else o[k] = 0u;
                }
                stop_any |= o[nout - 1];
                transpose32(o);
                const u64 word = (tile_base >> 5) + ((u64)(it * W + w) << 5) + lane;   // word index
                if ((word << 5) < states) {
                    srv_u64* dst = J->table + (word << 5);
                    for (u32 l = 0; l < lanes; l++) dst[l] = (srv_u64)o[l] | (1ull << 32);
                }
            }
            if (__any_sync(0xffffffffu, stop_any != 0u) && lane == 0) atomicOr(&J->st->any, 1u);
        }
    }
    if (kind == SRV_SAT) {
        u64 idx = ~0ull;
        if (first != 0xffffffffu) idx = tile_base + ((u64)(first >> 5) << 10) + ((u64)lane << 5) + (first & 31u);
        idx = warp_min(idx);
        cnt = __reduce_add_sync(0xffffffffu, cnt);
        if (lane == 0 && cnt) {
            atomicAdd(&J->st->count, (u64)cnt);
            atomicMin(&J->st->min_idx, idx);
        }
    } else if (kind == SRV_QSAT) {
        if (M < 10) {
            cand = warp_min(cand);
            if (lane == 0 && cand != ~0ull) atomicMin(&J->st->min_idx, cand);
        } else if (M < SRV_TILE_BITS) {
            const u32 y = tree_rt(acc, allbits, 10, (int)M - 10);
            const u32 d = (dec_all ? ~y : y) & unit_mask((int)M - 10);
            if (lane == 0 && d != 0u) atomicMin(&J->st->min_idx, (tile_base >> M) + ((__ffs(d) - 1) >> (M - 10)));
        } else {
            const u32 y = tree_rt(acc, allbits, 10, 5);
            if (lane == 0) vals[J->val_off + (tile - J->tile_begin)] = (uint8_t)(y & 1u);
        }
    }
    __syncwarp();
}

// The tile a job may hand out up to: its planned slice, or in the roll-over
// phase its next quarter slice, unless it has been decided already (lowest
// witness or decisive unit found).
__device__ __forceinline__ u64 claim_limit(const SrvJob* J, u32 phase) {
    if (!phase) return J->tile_end;
    if (!(J->flags & SRV_JOB_FIND_ALL) && J->kind != SRV_TABLE && *(volatile const u64*)&J->st->min_idx != ~0ull)
        return J->tile_end;
    return J->tile_hard;
}

// Hands out the job's next tile if it lies below `limit` (~0 otherwise).  A
// compare-and-swap, so the cursor never passes the limit and stays exact
// across epochs; a failed swap means another warp took a tile, so the loop
// ends after at most limit - cursor rounds.
__device__ __forceinline__ u64 claim_tile(SrvState* st, u64 limit) {
    u64 cur = *(volatile const u64*)&st->claim;
    while (cur < limit) {
        const u64 prev = atomicCAS(&st->claim, cur, cur + 1);
        if (prev == cur) return cur;
        cur = prev;
    }
    return ~0ull;
}

// One warp per CTA; the dynamic shared memory is max_slots * slot bytes.
// cls 0 serves the epoch's narrow jobs, cls 1 its wide ones.
template <int W, int G, bool DISPATCH>
__global__ void __launch_bounds__(32, 1) serve_epoch(const SrvEpoch* __restrict__ hdr, SrvJob* __restrict__ jobs,
                                                  uint8_t* __restrict__ vals, u32 cls) {
    extern __shared__ __align__(16) char smem[];
    const u32 n_narrow = hdr->n_narrow;
    const u32 njobs = cls == 0 ? n_narrow : hdr->njobs - n_narrow;
    if (cls != 0) jobs += n_narrow;
    const u32 lane = threadIdx.x & 31u;
    char* Sl = smem + lane * (W * 4);
    Dec dc;
    dc.km = hdr->hi_mul;
    dc.sb = hdr->slot_bytes;
    u32 j = njobs ? blockIdx.x % njobs : 0;
    u32 phase = 0;   // 0: the planned slices; 1: on into the next slices
    while (njobs) {
        // the job this warp is on: one claim, no search
        SrvJob* J = jobs + j;
        u64 tile = ~0ull;
        if (lane == 0) tile = claim_tile(J->st, claim_limit(J, phase));
        tile = __shfl_sync(0xffffffffu, tile, 0);
        if (tile == ~0ull) {
            // the next job after j (round robin) with a tile left below its
            // limit: 32 jobs per step, one per lane, so a pass over an epoch
            // of hundreds of jobs costs a few dependent L2 reads, not hundreds
            int pick = -1;
            for (u32 base = 1; base < njobs && pick < 0; base += 32) {
                const u32 k = base + lane;
                bool has = false;
                u32 jj = 0;
                if (k < njobs) {
                    jj = j + k;
                    if (jj >= njobs) jj -= njobs;
                    has = *(volatile const u64*)&jobs[jj].st->claim < claim_limit(&jobs[jj], phase);
                }
                const u32 m = __ballot_sync(0xffffffffu, has);
                if (m) pick = __shfl_sync(0xffffffffu, (int)jj, __ffs(m) - 1);
            }
            if (pick >= 0) {
                j = (u32)pick;   // claimed on the next turn (or found dry there)
            } else if (phase == 0) {
                phase = 1;       // job j itself is tried again at the new limit
            } else {
                break;
            }
            continue;
        }
        do_tile<W, G, DISPATCH>(J, tile, Sl, lane, vals, dc);
    }
}

typedef void (*EpochKernel)(const SrvEpoch*, SrvJob*, uint8_t*, u32);

// the instantiation of each shape of kSrvShapes, in order
EpochKernel kernel_of(uint32_t shape) {
    static const EpochKernel k[SRV_NSHAPES] = {
        serve_epoch<4, 4, false>, serve_epoch<4, 1, true>, serve_epoch<4, 2, true>,
        serve_epoch<4, 4, true>,  serve_epoch<2, 1, true>, serve_epoch<2, 2, true>,
    };
    return shape < SRV_NSHAPES ? k[shape] : nullptr;
}

}  // namespace

extern "C" int nsat_launch_serve_epoch(const SrvEpoch* hdr, SrvJob* jobs, uint32_t max_slots, uint8_t* vals,
                                       int grid, uint32_t cls, uint32_t shape, cudaStream_t stream) {
    // the dynamic shared memory limit was raised by nsat_serve_occupancy
    const EpochKernel fn = kernel_of(shape);
    if (!fn) return -1;
    const size_t smem = (size_t)max_slots * srv_slot_bytes(shape);
    fn<<<grid, 32, smem, stream>>>(hdr, jobs, vals, cls);
    return cudaGetLastError() == cudaSuccess ? 0 : -4;
}

extern "C" int nsat_serve_occupancy(uint32_t max_slots, uint32_t shape, int* ctas_per_sm) {
    const EpochKernel fn = kernel_of(shape);
    if (!fn || max_slots > SRV_MAX_SLOTS) return -1;
    const size_t smem = (size_t)max_slots * srv_slot_bytes(shape);
    // the limit covers every slot count, so launches captured earlier stay valid
    if (cudaFuncSetAttribute((const void*)fn, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             SRV_MAX_SLOTS * srv_slot_bytes(shape)) != cudaSuccess)
        return -4;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(ctas_per_sm, (const void*)fn, 32, smem) == cudaSuccess ? 0 : -4;
}

// device_template.cuh -- sm_100a kernels specialised per circuit by NVRTC.
//
// The host generator (codegen.cpp) prepends a prelude that defines:
//   constexpr ints NSAT_NIN, NSAT_NOUT, NSAT_NB (enumeration bits), NSAT_NT
//   (threads per CTA), NSAT_IT / NSAT_WB / NSAT_CB (log2 of iterations per
//   warp, warps per CTA and CTAs per launch), NSAT_BOUNDS (the kernels'
//   __launch_bounds__), NSAT_C (= 10+IT+WB+CB, log2 of
//   assignments per launch), NSAT_M (QSAT unit level), NSAT_Q0ALL,
//   NSAT_ALLBITS (bit j = quantifier of enumeration bit j is All),
//   NSAT_DATA (1 = items come from a buffer instead of the circuit),
//   NSAT_FMT (table entry format);
// and the generated device functions
//   nsat_inputs_fixed(x, lane, warp, cta, launch)  -- inputs that stay fixed
//   nsat_inputs_iter(x, it)                        -- inputs that follow `it`
//   nsat_eval1(x) -> u32          output 0 as a 32-lane word
//   nsat_eval_all(x, o)           all outputs (table mode)
//   nsat_inputs_word(x, w)        inputs of word index w (table mode)
//
// Assignment enumeration inside one launch (bit p of the launch-relative
// index selects circuit input IN_OF_BIT[p], baked into the functions above):
//   p 0..4   lane of the 32-bit word (constants 0xAAAAAAAA ... 0xFFFF0000)
//   p 5..9   lane of the warp
//   p 10..   iteration of the warp's loop (IT bits), warp in CTA (WB bits),
//            CTA in grid (CB bits); bits >= C come from the launch index.
// No input is ever read from memory: the kernels are pure ALU work plus a
// few bytes of results.

typedef unsigned int u32;
typedef unsigned long long u64;

struct LaunchOut {
    u64 min_idx;   // SAT: lowest satisfying launch-relative index; QSAT: lowest decisive unit
    u64 count;     // SAT: solutions in this launch
    u32 tree;      // QSAT: tree value of the launch when no unit boundary is inside it
    u32 ticket;    // CTAs finished (last-CTA tail), reset by the last CTA
    u32 any;       // table build: some STOP output seen
    u32 err;
};

__device__ __forceinline__ u64 warp_min_u64(u64 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        u64 w = __shfl_xor_sync(0xffffffffu, v, o);
        v = w < v ? w : v;
    }
    return v;
}

#if NSAT_MODE_SAT
// --------------------------------------------------------------------------
// SAT: count every satisfying assignment and find the lowest one.
extern "C" __global__ void NSAT_BOUNDS
nsat_sat(u64 launch, LaunchOut* __restrict__ out) {
    const u32 lane = threadIdx.x & 31u;
    const u32 warp = threadIdx.x >> 5;
    const u32 cta = blockIdx.x;
    u32 x[NSAT_NIN];
    nsat_inputs_fixed(x, lane, warp, cta, launch);
    u32 cnt = 0;
    u32 first_it = 0xffffffffu, first_bit = 0;
    for (u32 it = 0; it < (1u << NSAT_IT); it++) {
        nsat_inputs_iter(x, it);
        const u32 y = nsat_eval1(x);
        cnt += __popc(y);
        if (y != 0u && first_it == 0xffffffffu) { first_it = it; first_bit = __ffs(y) - 1; }
    }
    u64 idx = ~0ull;
    if (first_it != 0xffffffffu) {
        const u64 w = ((u64)cta << (5 + NSAT_IT + NSAT_WB)) | ((u64)warp << (5 + NSAT_IT)) |
                      ((u64)first_it << 5) | lane;
        idx = (w << 5) | first_bit;
    }
    idx = warp_min_u64(idx);
    cnt = __reduce_add_sync(0xffffffffu, cnt);
    if constexpr (NSAT_NT == 32) {
        if (lane == 0 && cnt != 0u) {
            atomicAdd(&out->count, (u64)cnt);
            atomicMin(&out->min_idx, idx);
        }
    } else {
        // one pair of atomics per CTA: launches with few iterations per warp
        // would otherwise queue every warp on the same two addresses
        // (a CTA counts at most 2^(10+IT+WB) <= 2^25 solutions)
        constexpr int NW = NSAT_NT / 32;
        __shared__ u64 s_idx[NW];
        __shared__ u32 s_cnt[NW];
        if (lane == 0) { s_idx[warp] = idx; s_cnt[warp] = cnt; }
        __syncthreads();
        if (warp == 0) {
            u64 ci = lane < (u32)NW ? s_idx[lane] : ~0ull;
            u32 cc = lane < (u32)NW ? s_cnt[lane] : 0u;
            ci = warp_min_u64(ci);
            cc = __reduce_add_sync(0xffffffffu, cc);
            if (lane == 0 && cc != 0u) {
                atomicAdd(&out->count, (u64)cc);
                atomicMin(&out->min_idx, ci);
            }
        }
    }
}
#endif

#if NSAT_MODE_QSAT
// --------------------------------------------------------------------------
// QSAT: AND/OR tree over the enumeration bits, innermost quantifier first.
// Nodes at level L cover 2^L consecutive items.  Units are the nodes at
// level M (one value of the first quantifier block each); a unit is
// decisive when its value differs from the first quantifier's identity
// (1 for Exists, 0 for All) and the lowest decisive unit is the witness.

template <int LVL, int CNT>
__device__ __forceinline__ u32 tree_up(u32 y) {
#pragma unroll
    for (int j = 0; j < CNT; j++) {
        if ((NSAT_ALLBITS >> (LVL + j)) & 1ull) y &= (y >> (1 << j));
        else y |= (y >> (1 << j));
    }
    return y;
}

__device__ __forceinline__ u32 tree_up_rt(u32 y, int lvl, int cnt) {
    for (int j = 0; j < cnt; j++) {
        if ((NSAT_ALLBITS >> (lvl + j)) & 1ull) y &= (y >> (1 << j));
        else y |= (y >> (1 << j));
    }
    return y;
}

// bits at multiples of 2^k inside a 32-bit node vector
__device__ __forceinline__ constexpr u32 unit_mask(int k) {
    return k == 0 ? 0xffffffffu : k == 1 ? 0x55555555u : k == 2 ? 0x11111111u
         : k == 3 ? 0x01010101u : k == 4 ? 0x00010001u : 0x1u;
}

// decisive unit positions among `nodes` node results whose units are 2^k nodes
__device__ __forceinline__ u32 decisive(u32 y, int k, int nodes) {
    const u32 valid = nodes >= 32 ? 0xffffffffu : ((1u << nodes) - 1u);
    return (NSAT_Q0ALL ? ~y : y) & unit_mask(k) & valid;
}

// number of consecutive levels from level 0 that share level 0's quantifier
__device__ constexpr int low_run(u64 allbits) {
    int k = 1;
    while (k < 64 && (((allbits >> k) ^ allbits) & 1ull) == 0ull) k++;
    return k;
}

extern "C" __global__ void NSAT_BOUNDS
nsat_qsat(u64 launch, LaunchOut* __restrict__ out, unsigned char* __restrict__ scratch,
          const u32* __restrict__ data) {
    constexpr int M = NSAT_M;
    // Folding.  When levels 0..9 (the word and the warp tile) and the lowest
    // FOLD iteration levels all carry level 0's quantifier and lie below the
    // units, their nodes are one AND (or OR) over 2^(10+FOLD) items, taken in
    // any order: a thread combines its words over 2^FOLD iterations with one
    // op per word, and a compare plus a warp vote gives the node at level
    // L0 = 10+FOLD.  Otherwise the word and tile trees run per iteration and
    // L0 = 10.  Stage 2 reduces the IT2 = IT-FOLD remaining iteration levels.
    constexpr int QLOW = low_run(NSAT_ALLBITS);
    constexpr bool FOLDED = M >= 10 && QLOW >= 10;
    constexpr int FOLD_CAP = QLOW < M ? QLOW : M;
    constexpr int FOLD = !FOLDED ? 0 : (FOLD_CAP < 10 + NSAT_IT ? FOLD_CAP : 10 + NSAT_IT) - 10;
    constexpr bool LOW_ALL = (NSAT_ALLBITS & 1ull) != 0ull;
    constexpr int L0 = 10 + FOLD;
    constexpr int IT2 = NSAT_IT - FOLD;
    constexpr int G1 = IT2 < 5 ? IT2 : 5;
    constexpr int G2 = IT2 - G1;
    const u32 lane = threadIdx.x & 31u;
    const u32 warp = threadIdx.x >> 5;
    const u32 cta = blockIdx.x;
    // launch-relative index of the first item of this warp's range
    const u64 warp_base = (((u64)cta << NSAT_WB) | warp) << (10 + NSAT_IT);
    u32 x[NSAT_NIN];
#if !NSAT_DATA
    nsat_inputs_fixed(x, lane, warp, cta, launch);
#endif
    u64 cand = ~0ull;      // lowest decisive unit seen by this thread (launch-relative)
    u32 acc1 = 0, acc2 = 0;
    u32 yacc = LOW_ALL ? 0xffffffffu : 0u;
    for (u32 it = 0; it < (1u << NSAT_IT); it++) {
#if NSAT_DATA
        const u64 gw = ((u64)launch << (NSAT_C - 5)) + ((warp_base + ((u64)it << 10)) >> 5) + lane;
        u32 y = data[gw];
#else
        nsat_inputs_iter(x, it);
        u32 y = nsat_eval1(x);
#endif
        u32 b, git;   // node value at level L0 (bit 0) and its index among the warp's L0 nodes
        if constexpr (FOLDED) {
            yacc = LOW_ALL ? (yacc & y) : (yacc | y);
            if (((it + 1u) & ((1u << FOLD) - 1u)) != 0u) continue;
            const bool v = LOW_ALL ? (yacc == 0xffffffffu) : (yacc != 0u);
            yacc = LOW_ALL ? 0xffffffffu : 0u;
            b = LOW_ALL ? (u32)__all_sync(0xffffffffu, v) : (u32)__any_sync(0xffffffffu, v);
            git = it >> FOLD;
        } else {
            const u64 tile_base = warp_base + ((u64)it << 10);   // first item of this warp tile
            // stage 0: the 32 lanes of the word (levels 0..4)
            if constexpr (M < 5) {
                y = tree_up<0, M>(y);
                const u32 d = decisive(y, M, 32);
                if (d != 0u && cand == ~0ull)
                    cand = ((tile_base + ((u64)lane << 5)) >> M) + (u64)((__ffs(d) - 1) >> M);
                continue;
            } else {
                y = tree_up<0, 5>(y);
            }
            // stage 1: the 32 words of the warp tile (levels 5..9)
            b = __ballot_sync(0xffffffffu, y & 1u);
            if constexpr (M >= 5 && M < 10) {
                b = tree_up<5, M - 5>(b);
                const u32 d = decisive(b, M - 5, 32);
                if (d != 0u && cand == ~0ull)
                    cand = (tile_base >> M) + (u64)((__ffs(d) - 1) >> (M - 5));
                continue;
            } else {
                b = tree_up<5, 5>(b);
            }
            git = it;
        }
        // stage 2: the warp's L0 nodes (levels L0..10+IT-1), 2^G1 at a time
        if constexpr (M >= L0 && IT2 > 0) {
            const u32 pos = git & ((1u << G1) - 1u);
            acc1 |= (b & 1u) << pos;
            if (pos == (1u << G1) - 1u) {
                const u64 grp_base = warp_base + ((u64)(git - pos) << L0);
                if constexpr (M < L0 + G1) {
                    const u32 y1 = tree_up<L0, M - L0>(acc1);
                    const u32 d = decisive(y1, M - L0, 1 << G1);
                    if (d != 0u && cand == ~0ull)
                        cand = (grp_base >> M) + (u64)((__ffs(d) - 1) >> (M - L0));
                } else {
                    const u32 y1 = tree_up<L0, G1>(acc1);
                    acc2 |= (y1 & 1u) << (git >> G1);
                }
                acc1 = 0;
            }
        } else if constexpr (M >= L0) {
            acc2 = b & 1u;   // IT2 == 0: one L0 node is the warp's whole range
        }
    }
    // stage 2b: groups of L0 nodes (levels L0+G1 .. 10+IT-1)
    u32 wres = 0;
    if constexpr (M >= L0 + G1 && IT2 > 0) {
        if constexpr (M < L0 + IT2) {
            const u32 y2 = tree_up<L0 + G1, M - L0 - G1>(acc2);
            const u32 d = decisive(y2, M - L0 - G1, 1 << G2);
            if (d != 0u && cand == ~0ull)
                cand = (warp_base >> M) + (u64)((__ffs(d) - 1) >> (M - L0 - G1));
        } else {
            wres = tree_up<L0 + G1, G2>(acc2) & 1u;
        }
    } else if constexpr (M >= L0 && IT2 == 0) {
        wres = acc2 & 1u;
    }
    // per-warp lowest candidate, one atomic per warp
    cand = warp_min_u64(cand);
    if (lane == 0 && cand != ~0ull) atomicMin(&out->min_idx, cand);
    // stage 3: warps of the CTA (levels 10+IT .. 10+IT+WB-1)
    if constexpr (M >= 10 + NSAT_IT) {
        __shared__ u32 s_res[32];
        __shared__ u32 s_last;
        if (lane == 0) s_res[warp] = wres;
        __syncthreads();
        u32 cres = 0;
        if (warp == 0) {
            u32 mbits = __ballot_sync(0xffffffffu, lane < (1u << NSAT_WB) ? s_res[lane] : 0u);
            const u64 cta_base = (u64)cta << (10 + NSAT_IT + NSAT_WB);
            if constexpr (M < 10 + NSAT_IT + NSAT_WB) {
                const u32 y3 = tree_up<10 + NSAT_IT, M - 10 - NSAT_IT>(mbits);
                const u32 d = decisive(y3, M - 10 - NSAT_IT, 1 << NSAT_WB);
                if (lane == 0 && d != 0u)
                    atomicMin(&out->min_idx, (cta_base >> M) + (u64)((__ffs(d) - 1) >> (M - 10 - NSAT_IT)));
            } else {
                cres = tree_up<10 + NSAT_IT, NSAT_WB>(mbits) & 1u;
            }
        }
        // stage 4: CTAs of the launch (levels 10+IT+WB .. C-1), last-CTA tail
        if constexpr (M >= 10 + NSAT_IT + NSAT_WB) {
            if constexpr (NSAT_CB == 0) {
                if (threadIdx.x == 0) out->tree = cres;
            } else {
                if (threadIdx.x == 0) {
                    scratch[cta] = (unsigned char)cres;
                    __threadfence();
                    const u32 t = atomicAdd(&out->ticket, 1u);
                    s_last = (t == (1u << NSAT_CB) - 1u) ? 1u : 0u;
                }
                __syncthreads();
                if (s_last) {
                    __threadfence();
                    int lvl = 10 + NSAT_IT + NSAT_WB;
                    int nodes = 1 << NSAT_CB;
                    unsigned char* src = scratch;
                    unsigned char* dst = scratch + (1 << NSAT_CB);
                    const int nw = NSAT_NT / 32;
                    bool done = false;
                    while (!done) {
                        const int k = nodes >= 32 ? 5 : (31 - __clz(nodes));   // log2(nodes) if < 32
                        const int groups = nodes >> k;
                        const bool units_here = M < lvl + k;
                        for (int gi = (int)warp; gi < groups; gi += nw) {
                            const int node = (gi << k) + (int)lane;
                            u32 v = (lane < (1u << k)) ? (u32)__ldcg(src + node) : 0u;
                            u32 mb = __ballot_sync(0xffffffffu, v & 1u);
                            if (units_here) {
                                const int ku = M - lvl;
                                mb = tree_up_rt(mb, lvl, ku);
                                const u32 d = decisive(mb, ku, 1 << k);
                                if (lane == 0 && d != 0u)
                                    atomicMin(&out->min_idx,
                                              ((((u64)gi << k) << lvl) >> M) + (u64)((__ffs(d) - 1) >> ku));
                            } else {
                                mb = tree_up_rt(mb, lvl, k);
                                if (lane == 0) dst[gi] = (unsigned char)(mb & 1u);
                            }
                        }
                        __syncthreads();
                        if (units_here) { done = true; break; }
                        lvl += k;
                        nodes = groups;
                        unsigned char* tmp = src; src = dst; dst = tmp;
                        if (nodes == 1) {
                            if (threadIdx.x == 0) out->tree = (u32)__ldcg(src);
                            done = true;
                        }
                    }
                    if (threadIdx.x == 0) out->ticket = 0u;
                }
            }
        }
    }
}
#endif

#if NSAT_MODE_TABLE
// --------------------------------------------------------------------------
// SATOSTOP next-state table: entry[s] = next(s) | STOP(s) << n.
// One thread evaluates 32 states bit-sliced, then transposes the 32x32 bit
// matrix (rows = outputs, columns = lanes) into per-state entries.

__device__ __forceinline__ void transpose32(u32* a) {
    // block-swap transpose: after the step for size j, row k and row k+j
    // exchange their off-diagonal j x j blocks
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

extern "C" __global__ void NSAT_BOUNDS
nsat_table(u64 nwords, u64 w0, void* __restrict__ table, LaunchOut* __restrict__ out) {
    // entries of words w0 .. w0+nwords-1 (32 states each), stored from table[0]
    const u64 stride = (u64)gridDim.x * NSAT_NT;
    u32 anystop = 0;
    for (u64 w = (u64)blockIdx.x * NSAT_NT + threadIdx.x; w < nwords; w += stride) {
        u32 x[NSAT_NIN];
        nsat_inputs_word(x, w0 + w);
        u32 o[64];
#pragma unroll
        for (int k = 0; k < 64; k++) o[k] = 0u;
        nsat_eval_all(x, o);
        anystop |= o[NSAT_NOUT - 1];
        constexpr int lanes = NSAT_NB >= 5 ? 32 : (1 << NSAT_NB);
#if NSAT_FMT == 0
        transpose32(o);
        uint4* dst = reinterpret_cast<uint4*>(reinterpret_cast<u32*>(table) + (w << 5));
        if (lanes == 32) {
#pragma unroll
            for (int q = 0; q < 8; q++) __stcs(dst + q, make_uint4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]));
        } else {
            for (int l = 0; l < lanes; l++) reinterpret_cast<u32*>(table)[l] = o[l];
        }
#else
        transpose32(o);
        if (NSAT_NOUT > 32) transpose32(o + 32);
        u64* t64 = reinterpret_cast<u64*>(table) + (w << 5);
#if NSAT_FMT == 2
        const u64 hi_or = 1ull << 32;   // distance 1 per entry
#else
        const u64 hi_or = 0ull;
#endif
        if (lanes == 32) {
            ulonglong2* dst = reinterpret_cast<ulonglong2*>(t64);
#pragma unroll
            for (int q = 0; q < 16; q++) {
                ulonglong2 v;
                v.x = (u64)o[2 * q] | ((u64)o[32 + 2 * q] << 32) | hi_or;
                v.y = (u64)o[2 * q + 1] | ((u64)o[32 + 2 * q + 1] << 32) | hi_or;
                __stcs(dst + q, v);
            }
        } else {
            for (int l = 0; l < lanes; l++) t64[l] = (u64)o[l] | ((u64)o[32 + l] << 32) | hi_or;
        }
#endif
    }
    if (__any_sync(0xffffffffu, anystop != 0u) && (threadIdx.x & 31u) == 0) atomicOr(&out->any, 1u);
}
#endif

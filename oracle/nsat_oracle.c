/*
 * nsat_oracle.c -- CPU restatement of the reference's solver semantics.
 *
 * TEST INFRASTRUCTURE ONLY: the checker for the CUDA path and the timed CPU
 * baseline.  The product library never links it (see nsat_oracle.h).
 *
 * The reference evaluates circuits through the external `gatenative` 0.2.0
 * crate (Cargo.toml:29), which is not vendored.  Its CPU path generates
 * bit-sliced C over machine words with `elem` inputs enumerated inside a call
 * and `arg` inputs fixed per call (main.rs:106-155).  This file restates that
 * as a slot-allocated bit-sliced interpreter over blocks of 8 x 64-bit words
 * (512 assignments), parallelised with OpenMP across blocks.
 */
#include "nsat_oracle.h"

#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define BW 8                 /* 64-bit words per block */
#define BLOCK_BITS 9         /* log2(64 * BW) */

static inline uint64_t gate_fn(uint32_t f, uint64_t a, uint64_t b) {
    switch (f) {
    case 0: return a & b;          /* And   */
    case 1: return ~(a | b);       /* Nor   */
    case 2: return a & ~b;         /* Nimpl */
    default: return a ^ b;         /* Xor   */
    }
}

static int check_circuit(const or_circuit* c) {
    if (!c || c->n == 0 || c->n > 128) return -1;
    for (uint32_t k = 0; k < c->g; k++) {
        if (c->gates[3 * k] > 3) return -1;
        if (c->gates[3 * k + 1] >= c->n + k || c->gates[3 * k + 2] >= c->n + k) return -1;
    }
    for (uint32_t j = 0; j < c->o; j++)
        if (c->outputs[2 * j] >= c->n + c->g) return -1;
    return 0;
}

int or_eval_scalar(const or_circuit* c, const uint8_t* in, uint8_t* out) {
    if (check_circuit(c)) return -1;
    uint8_t* w = (uint8_t*)malloc(c->n + c->g);
    if (!w) return -2;
    for (uint32_t i = 0; i < c->n; i++) w[i] = in[i] & 1;
    for (uint32_t k = 0; k < c->g; k++)
        w[c->n + k] = (uint8_t)(gate_fn(c->gates[3 * k], w[c->gates[3 * k + 1]],
                                        w[c->gates[3 * k + 2]]) & 1);
    for (uint32_t j = 0; j < c->o; j++)
        out[j] = w[c->outputs[2 * j]] ^ (c->outputs[2 * j + 1] & 1);
    free(w);
    return 0;
}

int or_eval_words(const or_circuit* c, const uint64_t* in, uint64_t* out) {
    if (check_circuit(c)) return -1;
    uint64_t* w = (uint64_t*)malloc(sizeof(uint64_t) * (c->n + c->g));
    if (!w) return -2;
    memcpy(w, in, sizeof(uint64_t) * c->n);
    for (uint32_t k = 0; k < c->g; k++)
        w[c->n + k] = gate_fn(c->gates[3 * k], w[c->gates[3 * k + 1]], w[c->gates[3 * k + 2]]);
    for (uint32_t j = 0; j < c->o; j++)
        out[j] = w[c->outputs[2 * j]] ^ (c->outputs[2 * j + 1] ? ~0ull : 0ull);
    free(w);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Slot-allocated program: dead gates dropped, wires mapped to reusable slots */

typedef struct { uint32_t f, d, a, b; } op_t;
typedef struct {
    uint32_t n, o, nslots, nops;
    op_t* ops;
    uint32_t* in_slot;   /* per input, UINT32_MAX if unused */
    uint32_t* out_slot;  /* per output */
    uint64_t* out_neg;   /* per output: xor mask */
} prog_t;

static void prog_free(prog_t* p) {
    free(p->ops); free(p->in_slot); free(p->out_slot); free(p->out_neg);
    memset(p, 0, sizeof(*p));
}

static int prog_build(const or_circuit* c, prog_t* p) {
    memset(p, 0, sizeof(*p));
    if (check_circuit(c)) return -1;
    uint32_t W = c->n + c->g;
    uint8_t* live = (uint8_t*)calloc(W, 1);
    int64_t* last = (int64_t*)malloc(sizeof(int64_t) * W);   /* last use position */
    uint32_t* slot = (uint32_t*)malloc(sizeof(uint32_t) * W);
    uint32_t* freelist = (uint32_t*)malloc(sizeof(uint32_t) * (W + 1));
    p->ops = (op_t*)malloc(sizeof(op_t) * (c->g + 1));
    p->in_slot = (uint32_t*)malloc(sizeof(uint32_t) * c->n);
    p->out_slot = (uint32_t*)malloc(sizeof(uint32_t) * (c->o + 1));
    p->out_neg = (uint64_t*)malloc(sizeof(uint64_t) * (c->o + 1));
    if (!live || !last || !slot || !freelist || !p->ops || !p->in_slot || !p->out_slot || !p->out_neg) {
        free(live); free(last); free(slot); free(freelist); prog_free(p);
        return -2;
    }
    for (uint32_t j = 0; j < c->o; j++) live[c->outputs[2 * j]] = 1;
    for (int64_t k = (int64_t)c->g - 1; k >= 0; k--)
        if (live[c->n + k]) { live[c->gates[3 * k + 1]] = 1; live[c->gates[3 * k + 2]] = 1; }
    /* last use: gate position k (0..g-1); outputs use position g */
    for (uint32_t i = 0; i < W; i++) last[i] = -1;
    for (uint32_t k = 0; k < c->g; k++) if (live[c->n + k]) {
        last[c->gates[3 * k + 1]] = k; last[c->gates[3 * k + 2]] = k;
    }
    for (uint32_t j = 0; j < c->o; j++) last[c->outputs[2 * j]] = c->g;
    uint32_t nfree = 0, nslots = 0;
    for (uint32_t i = 0; i < c->n; i++) {
        if (live[i]) { slot[i] = nslots++; p->in_slot[i] = slot[i]; }
        else p->in_slot[i] = UINT32_MAX;
    }
    uint32_t nops = 0;
    for (uint32_t k = 0; k < c->g; k++) {
        uint32_t w = c->n + k;
        if (!live[w]) continue;
        uint32_t a = c->gates[3 * k + 1], b = c->gates[3 * k + 2];
        /* allocate destination before freeing operands: slots never alias a
         * source of the same op */
        uint32_t d = nfree ? freelist[--nfree] : nslots++;
        slot[w] = d;
        p->ops[nops].f = c->gates[3 * k]; p->ops[nops].d = d;
        p->ops[nops].a = slot[a]; p->ops[nops].b = slot[b];
        nops++;
        if (last[a] == (int64_t)k) { freelist[nfree++] = slot[a]; last[a] = -2; }
        if (b != a && last[b] == (int64_t)k) { freelist[nfree++] = slot[b]; last[b] = -2; }
    }
    for (uint32_t j = 0; j < c->o; j++) {
        p->out_slot[j] = slot[c->outputs[2 * j]];
        p->out_neg[j] = c->outputs[2 * j + 1] ? ~0ull : 0ull;
    }
    p->n = c->n; p->o = c->o; p->nslots = nslots ? nslots : 1; p->nops = nops;
    free(live); free(last); free(slot); free(freelist);
    return 0;
}

/* Evaluate one block of 512 assignments.  pos[i] = enumeration bit that drives
 * input i; assignment index = (blk << 9) | (k << 6) | l for word k, lane l.
 * S is nslots*BW scratch.  Outputs land in out[j*BW + k]. */
static const uint64_t LANE_PAT[6] = {
    0xAAAAAAAAAAAAAAAAull, 0xCCCCCCCCCCCCCCCCull, 0xF0F0F0F0F0F0F0F0ull,
    0xFF00FF00FF00FF00ull, 0xFFFF0000FFFF0000ull, 0xFFFFFFFF00000000ull};

static void prog_eval_block(const prog_t* p, const uint32_t* pos, uint64_t blk,
                            const uint64_t* hi_bits, uint64_t* S, uint64_t* out) {
    for (uint32_t i = 0; i < p->n; i++) {
        uint32_t s = p->in_slot[i];
        if (s == UINT32_MAX) continue;
        uint32_t b = pos[i];
        uint64_t* d = S + (size_t)s * BW;
        if (b < 6) {
            for (int k = 0; k < BW; k++) d[k] = LANE_PAT[b];
        } else if (b < BLOCK_BITS) {
            for (int k = 0; k < BW; k++) d[k] = ((k >> (b - 6)) & 1) ? ~0ull : 0ull;
        } else {
            uint32_t bb = b - BLOCK_BITS;
            uint64_t v = bb < 64 ? ((blk >> bb) & 1) : ((hi_bits[(bb - 64) >> 6] >> ((bb - 64) & 63)) & 1);
            for (int k = 0; k < BW; k++) d[k] = v ? ~0ull : 0ull;
        }
    }
    for (uint32_t t = 0; t < p->nops; t++) {
        const op_t* op = &p->ops[t];
        uint64_t* d = S + (size_t)op->d * BW;
        const uint64_t* a = S + (size_t)op->a * BW;
        const uint64_t* b = S + (size_t)op->b * BW;
        switch (op->f) {
        case 0: for (int k = 0; k < BW; k++) d[k] = a[k] & b[k]; break;
        case 1: for (int k = 0; k < BW; k++) d[k] = ~(a[k] | b[k]); break;
        case 2: for (int k = 0; k < BW; k++) d[k] = a[k] & ~b[k]; break;
        default: for (int k = 0; k < BW; k++) d[k] = a[k] ^ b[k]; break;
        }
    }
    for (uint32_t j = 0; j < p->o; j++) {
        const uint64_t* s = S + (size_t)p->out_slot[j] * BW;
        for (int k = 0; k < BW; k++) out[j * BW + k] = s[k] ^ p->out_neg[j];
    }
}

static int set_threads(int threads) {
#ifdef _OPENMP
    return threads > 0 ? threads : omp_get_max_threads();
#else
    (void)threads;
    return 1;
#endif
}

/* ---------------------------------- SAT ---------------------------------- */

int or_sat_range(const or_circuit* c, uint64_t begin, uint64_t end, int threads,
                 uint64_t* count, uint64_t* lowest) {
    if (check_circuit(c) || c->o < 1 || c->n > 63) return -1;
    uint64_t total = 1ull << c->n;
    if (begin > end || end > total) return -1;
    *count = 0; *lowest = UINT64_MAX;
    if (begin == end) return 0;
    if (c->n < BLOCK_BITS + 1) {
        uint8_t in[64], out;
        or_circuit c1 = *c; c1.o = 1;
        for (uint64_t v = begin; v < end; v++) {
            for (uint32_t b = 0; b < c->n; b++) in[b] = (v >> b) & 1;
            or_eval_scalar(&c1, in, &out);
            if (out) { (*count)++; if (*lowest == UINT64_MAX) *lowest = v; }
        }
        return 0;
    }
    or_circuit c1 = *c; c1.o = 1;
    prog_t p;
    if (prog_build(&c1, &p)) return -2;
    uint32_t pos[128];
    for (uint32_t i = 0; i < c->n; i++) pos[i] = i;
    uint64_t b0 = begin >> BLOCK_BITS, b1 = (end + 511) >> BLOCK_BITS;
    uint64_t gcount = 0, glow = UINT64_MAX;
    int nt = set_threads(threads);
    int err = 0;
#pragma omp parallel num_threads(nt) reduction(+ : gcount) reduction(min : glow)
    {
        uint64_t* S = (uint64_t*)malloc(sizeof(uint64_t) * p.nslots * BW);
        uint64_t out[BW];
        if (!S) {
#pragma omp atomic write
            err = 1;
        } else {
#pragma omp for schedule(dynamic, 64)
            for (uint64_t blk = b0; blk < b1; blk++) {
                prog_eval_block(&p, pos, blk, NULL, S, out);
                for (int k = 0; k < BW; k++) {
                    uint64_t w = out[k];
                    uint64_t base = (blk << BLOCK_BITS) | ((uint64_t)k << 6);
                    /* clip to [begin, end) */
                    if (base + 64 <= begin || base >= end) continue;
                    if (base < begin) w &= ~0ull << (begin - base);
                    if (base + 64 > end) w &= (end - base) >= 64 ? ~0ull : ((1ull << (end - base)) - 1);
                    if (w) {
                        gcount += (uint64_t)__builtin_popcountll(w);
                        uint64_t v = base + (uint64_t)__builtin_ctzll(w);
                        if (v < glow) glow = v;
                    }
                }
            }
            free(S);
        }
    }
    prog_free(&p);
    if (err) return -2;
    *count = gcount; *lowest = glow;
    return 0;
}

/* ----------------------------- QuantReducer ------------------------------ */
/* Restates qsat.rs:172-291.  quants are stored reversed (index 0 = the last
 * input, i.e. the lowest bit of the item index), All = 1, Exists = 0. */

struct or_qr {
    int nq;
    uint8_t q[64];      /* reversed quantifiers */
    uint8_t r[64];      /* per-level partial results */
    int started;
    uint64_t start, all_mask, first_mask, other_mask;
    int has_solution;
    uint64_t solution;
    /* min-heap of (index, item) for out-of-order pushes */
    uint64_t* hidx;
    uint8_t* hitem;
    size_t hlen, hcap;
};

or_qr* or_qr_new(const uint8_t* quants, int nq) {
    if (nq < 1 || nq > 64) return NULL;
    or_qr* qr = (or_qr*)calloc(1, sizeof(or_qr));
    if (!qr) return NULL;
    qr->nq = nq;
    int fb = 0;
    while (fb < nq && (quants[fb] & 1) == (quants[0] & 1)) fb++;
    for (int i = 0; i < nq; i++) { qr->q[i] = quants[nq - 1 - i] & 1; qr->r[i] = qr->q[i]; }
    qr->all_mask = nq == 64 ? ~0ull : ((1ull << nq) - 1);
    uint64_t fm = fb == 64 ? ~0ull : ((1ull << fb) - 1);
    qr->first_mask = (nq - fb) >= 64 ? 0 : fm << (nq - fb);
    qr->other_mask = qr->all_mask & ~qr->first_mask;
    return qr;
}

void or_qr_free(or_qr* qr) {
    if (!qr) return;
    free(qr->hidx); free(qr->hitem); free(qr);
}

static int qr_is_end(const or_qr* qr) { return qr->started && (qr->start & qr->all_mask) == 0; }

static void qr_apply(or_qr* qr, int item) {
    qr->started = 1;
    uint64_t index = qr->start;
    int prev = item & 1;
    for (int i = 0; i < qr->nq; i++) {
        int q = qr->q[i], r = qr->r[i];
        prev = (r & prev) | ((r ^ prev) & !q);
        qr->r[i] = (uint8_t)prev;
        if ((index & 1) == 0) break;
        index >>= 1;
        qr->r[i] = (uint8_t)q;
    }
    if (!qr->has_solution && (qr->start & qr->other_mask) == qr->other_mask &&
        (prev ^ qr->q[qr->nq - 1])) {
        int fb = __builtin_popcountll(qr->first_mask);
        /* first-block value, bit-reversed into input order (bit k = input k) */
        uint64_t v = qr->start >> (qr->nq - fb);
        uint64_t rev = 0;
        for (int k = 0; k < fb; k++) rev |= ((v >> k) & 1) << (fb - 1 - k);
        qr->has_solution = 1;
        qr->solution = rev;
    }
    qr->start += 1;
}

static void heap_push(or_qr* qr, uint64_t idx, uint8_t item) {
    if (qr->hlen == qr->hcap) {
        size_t nc = qr->hcap ? qr->hcap * 2 : 64;
        qr->hidx = (uint64_t*)realloc(qr->hidx, nc * sizeof(uint64_t));
        qr->hitem = (uint8_t*)realloc(qr->hitem, nc);
        qr->hcap = nc;
    }
    size_t i = qr->hlen++;
    while (i > 0) {
        size_t par = (i - 1) / 2;
        if (qr->hidx[par] <= idx) break;
        qr->hidx[i] = qr->hidx[par]; qr->hitem[i] = qr->hitem[par];
        i = par;
    }
    qr->hidx[i] = idx; qr->hitem[i] = item;
}

static void heap_pop(or_qr* qr) {
    uint64_t idx = qr->hidx[--qr->hlen];
    uint8_t item = qr->hitem[qr->hlen];
    size_t i = 0, n = qr->hlen;
    for (;;) {
        size_t l = 2 * i + 1, r = l + 1, m = i;
        uint64_t mv = idx;
        if (l < n && qr->hidx[l] < mv) { m = l; mv = qr->hidx[l]; }
        if (r < n && qr->hidx[r] < mv) { m = r; }
        if (m == i) break;
        qr->hidx[i] = qr->hidx[m]; qr->hitem[i] = qr->hitem[m];
        i = m;
    }
    if (n) { qr->hidx[i] = idx; qr->hitem[i] = item; }
}

int or_qr_push(or_qr* qr, uint64_t index, int item) {
    if (qr_is_end(qr)) return -1;
    heap_push(qr, index, (uint8_t)(item & 1));
    /* flush (qsat.rs:252-272): apply items while the heap top is the next
     * index; stop right after the apply that produced the solution */
    while (qr->hlen && qr->hidx[0] == qr->start) {
        int old = qr->has_solution;
        int it = qr->hitem[0];
        heap_pop(qr);
        qr_apply(qr, it);
        if (!old && qr->has_solution) break;
        if (qr_is_end(qr)) break;
    }
    return 0;
}

/* the items of packed words (item k = bit k%32 of word k/32), in index order,
 * until the reducer is final; test helper for the device reduction */
int or_qr_push_words(or_qr* qr, const uint32_t* words, uint64_t nwords) {
    return or_qr_push_words_from(qr, 0, words, nwords);
}

/* Items first .. first + 32 nwords - 1: item first + k is bit k % 32 of
 * word k / 32 (consecutive batches of one item sequence). */
int or_qr_push_words_from(or_qr* qr, uint64_t first, const uint32_t* words, uint64_t nwords) {
    for (uint64_t k = 0; k < nwords * 32u; k++) {
        if (qr_is_end(qr) || qr->has_solution) break;
        if (or_qr_push(qr, first + k, (int)((words[k >> 5] >> (k & 31u)) & 1u))) return -1;
    }
    return 0;
}

int or_qr_final(const or_qr* qr, int* reversed, uint32_t* solution_bits,
                int* has_solution, uint64_t* solution) {
    if (!(qr_is_end(qr) || qr->has_solution)) return 0;
    *reversed = qr->q[qr->nq - 1];
    *solution_bits = (uint32_t)__builtin_popcountll(qr->first_mask);
    *has_solution = qr->has_solution;
    *solution = qr->has_solution ? qr->solution : 0;
    return 1;
}

/* --------------------------------- QSAT ---------------------------------- */

static int first_block_len(const uint8_t* q, int n) {
    int f = 0;
    while (f < n && (q[f] & 1) == (q[0] & 1)) f++;
    return f;
}

/* Evaluate the circuit in v-order for item indices [v0, v0 + 2^len) and push
 * every value into qr (indices relative to v0). */
static int qsat_push_range(const prog_t* p, uint32_t n, uint64_t v0, uint32_t len,
                           or_qr* qr, uint64_t* S) {
    uint32_t pos[128];
    for (uint32_t i = 0; i < n; i++) pos[i] = n - 1 - i;
    uint64_t out[BW];
    uint64_t items = 1ull << len;
    for (uint64_t rel = 0; rel < items; rel += 512) {
        uint64_t blk = (v0 + rel) >> BLOCK_BITS;
        prog_eval_block(p, pos, blk, NULL, S, out);
        for (int k = 0; k < BW; k++) {
            for (int l = 0; l < 64; l++) {
                uint64_t idx = rel + (uint64_t)k * 64 + l;
                if (or_qr_push(qr, idx, (int)((out[k] >> l) & 1))) return 0;
                int rv; uint32_t sb; int hs; uint64_t sol;
                (void)rv; (void)sb; (void)sol;
                if (or_qr_final(qr, &rv, &sb, &hs, &sol) && hs) return 0;
            }
        }
    }
    return 0;
}

int or_qsat(const or_circuit* c, const uint8_t* quants, int mode, int threads,
            int* reversed, uint32_t* solution_bits, int* has_solution,
            uint64_t* solution) {
    if (check_circuit(c) || c->o < 1 || c->n > 40) return -1;
    const uint32_t n = c->n;
    const int f = first_block_len(quants, (int)n);
    if (n < BLOCK_BITS + 2) {
        /* scalar path of qsat.rs:1991-1998 */
        or_qr* qr = or_qr_new(quants, (int)n);
        or_circuit c1 = *c; c1.o = 1;
        uint8_t in[64], out;
        for (uint64_t v = 0; v < (1ull << n); v++) {
            for (uint32_t i = 0; i < n; i++) in[i] = (v >> (n - 1 - i)) & 1;
            or_eval_scalar(&c1, in, &out);
            or_qr_push(qr, v, out);
        }
        int ok = or_qr_final(qr, reversed, solution_bits, has_solution, solution);
        or_qr_free(qr);
        return ok ? 0 : -3;
    }
    or_circuit c1 = *c; c1.o = 1;
    prog_t p;
    if (prog_build(&c1, &p)) return -2;
    int rc = 0;
    if (mode == 0) {
        or_qr* qr = or_qr_new(quants, (int)n);
        uint64_t* S = (uint64_t*)malloc(sizeof(uint64_t) * p.nslots * BW);
        qsat_push_range(&p, n, 0, n, qr, S);
        if (!or_qr_final(qr, reversed, solution_bits, has_solution, solution)) rc = -3;
        free(S);
        or_qr_free(qr);
        prog_free(&p);
        return rc;
    }
    /* chunked: top t bits select a chunk; each chunk is a sub-tree over the
     * remaining n-t inputs reduced by its own QuantReducer */
    uint32_t t = n - (BLOCK_BITS + 1);
    if (t > 12) t = 12;
    uint32_t len = n - t;
    uint64_t nch = 1ull << t;
    uint8_t* val = (uint8_t*)malloc(nch);
    uint8_t* has = (uint8_t*)malloc(nch);
    uint64_t* sub = (uint64_t*)malloc(sizeof(uint64_t) * nch);
    int nt = set_threads(threads);
#pragma omp parallel num_threads(nt)
    {
        uint64_t* S = (uint64_t*)malloc(sizeof(uint64_t) * p.nslots * BW);
#pragma omp for schedule(dynamic, 1)
        for (uint64_t ch = 0; ch < nch; ch++) {
            or_qr* qr = or_qr_new(quants + t, (int)len);
            qsat_push_range(&p, n, ch << len, len, qr, S);
            int rv, hs; uint32_t sb; uint64_t sol;
            or_qr_final(qr, &rv, &sb, &hs, &sol);
            /* tree value of the sub-formula: solution found XOR first quant All
             * (qsat.rs:1165-1170) */
            val[ch] = (uint8_t)((hs ? 1 : 0) ^ rv);
            has[ch] = (uint8_t)hs;
            sub[ch] = sol;
            or_qr_free(qr);
        }
        free(S);
    }
    or_qr* top = or_qr_new(quants, (int)t);
    int done = 0;
    for (uint64_t ch = 0; ch < nch && !done; ch++) {
        or_qr_push(top, ch, val[ch]);
        int rv, hs; uint32_t sb; uint64_t sol;
        if (or_qr_final(top, &rv, &sb, &hs, &sol)) {
            done = 1;
            *reversed = rv;
            *solution_bits = (uint32_t)f;
            *has_solution = hs;
            if (hs && (uint32_t)f > t) {
                /* FinalResult::join (qsat.rs:108-140): chunk witness supplies
                 * the first-block bits below the top t */
                uint64_t chunk = ch;   /* the reducer stopped at this chunk */
                uint64_t low = sub[chunk];
                uint64_t full = sol | (low << t);
                *solution = f >= 64 ? full : (full & ((1ull << f) - 1));
            } else {
                *solution = hs ? sol : 0;
            }
        }
    }
    if (!done) rc = -3;
    or_qr_free(top);
    free(val); free(has); free(sub);
    prog_free(&p);
    return rc;
}

/* ------------------------------- SATOSTOP -------------------------------- */

int or_stop_table(const or_circuit* c, int threads, uint64_t* table) {
    if (check_circuit(c) || c->o != c->n + 1 || c->n > 32 || c->n < 1) return -1;
    const uint32_t n = c->n;
    if (n < BLOCK_BITS) {
        uint8_t in[64], out[65];
        for (uint64_t s = 0; s < (1ull << n); s++) {
            for (uint32_t b = 0; b < n; b++) in[b] = (s >> b) & 1;
            or_eval_scalar(c, in, out);
            uint64_t v = 0;
            for (uint32_t b = 0; b <= n; b++) v |= (uint64_t)out[b] << b;
            table[s] = v;
        }
        return 0;
    }
    prog_t p;
    if (prog_build(c, &p)) return -2;
    uint32_t pos[128];
    for (uint32_t i = 0; i < n; i++) pos[i] = i;
    uint64_t nblk = 1ull << (n - BLOCK_BITS);
    int nt = set_threads(threads);
#pragma omp parallel num_threads(nt)
    {
        uint64_t* S = (uint64_t*)malloc(sizeof(uint64_t) * p.nslots * BW);
        uint64_t* out = (uint64_t*)malloc(sizeof(uint64_t) * (n + 1) * BW);
#pragma omp for schedule(static)
        for (uint64_t blk = 0; blk < nblk; blk++) {
            prog_eval_block(&p, pos, blk, NULL, S, out);
            for (int k = 0; k < BW; k++)
                for (int l = 0; l < 64; l++) {
                    uint64_t v = 0;
                    for (uint32_t j = 0; j <= n; j++) v |= ((out[j * BW + k] >> l) & 1) << j;
                    table[(blk << BLOCK_BITS) | ((uint64_t)k << 6) | (uint64_t)l] = v;
                }
        }
        free(S); free(out);
    }
    prog_free(&p);
    return 0;
}

int or_stop_solve(uint32_t n, uint32_t u, const uint64_t* table, int mode,
                  int threads, int* found, uint64_t* start, uint64_t* end,
                  uint64_t* steps, uint32_t* rounds) {
    if (n < 1 || n > 32 || u > n) return -1;
    *found = 0; *start = *end = *steps = 0; *rounds = 0;
    const uint64_t N = 1ull << n;
    const uint64_t nmask = N - 1;
    const uint64_t stopbit = 1ull << n;
    const uint64_t step = 1ull << (n - u);
    uint64_t* nx = (uint64_t*)malloc(sizeof(uint64_t) * N);
    uint64_t* nx2 = (uint64_t*)malloc(sizeof(uint64_t) * N);
    uint64_t* ds = (uint64_t*)malloc(sizeof(uint64_t) * N);
    uint64_t* ds2 = (uint64_t*)malloc(sizeof(uint64_t) * N);
    if (!nx || !nx2 || !ds || !ds2) { free(nx); free(nx2); free(ds); free(ds2); return -2; }
    int nt = set_threads(threads);
    int any_stop = 0;
#pragma omp parallel for num_threads(nt) reduction(| : any_stop)
    for (uint64_t s = 0; s < N; s++) {
        nx[s] = table[s] & (nmask | stopbit);
        ds[s] = 1;
        if (table[s] & stopbit) any_stop = 1;
    }
    if (any_stop) {
        uint64_t best = UINT64_MAX;
        for (uint32_t r = 1; r <= n; r++) {
#pragma omp parallel for num_threads(nt)
            for (uint64_t s = 0; s < N; s++) {
                uint64_t v = nx[s];
                if (v & stopbit) { nx2[s] = v; ds2[s] = ds[s]; }
                else {
                    uint64_t t = v & nmask;
                    nx2[s] = nx[t];
                    ds2[s] = ds[s] + ds[t];
                }
            }
            uint64_t* tp = nx; nx = nx2; nx2 = tp;
            tp = ds; ds = ds2; ds2 = tp;
            *rounds = r;
            for (uint64_t k = 0; k < (1ull << u); k++) {
                uint64_t s = k * step;
                if (nx[s] & stopbit) { best = s; break; }
            }
            if (best != UINT64_MAX && (mode == 0 || best == 0)) break;
        }
        if (best != UINT64_MAX) {
            *found = 1; *start = best; *end = nx[best] & nmask; *steps = ds[best];
        }
    }
    free(nx); free(nx2); free(ds); free(ds2);
    return 0;
}

int or_stop_replay(const or_circuit* c, uint64_t s0, uint64_t max_steps,
                   uint64_t* end, uint64_t* steps) {
    if (check_circuit(c) || c->o != c->n + 1 || c->n > 63) return -1;
    uint8_t in[64], out[65];
    uint64_t s = s0;
    for (uint64_t k = 1; k <= max_steps; k++) {
        for (uint32_t b = 0; b < c->n; b++) in[b] = (s >> b) & 1;
        or_eval_scalar(c, in, out);
        uint64_t nxt = 0;
        for (uint32_t b = 0; b < c->n; b++) nxt |= (uint64_t)out[b] << b;
        s = nxt;
        if (out[c->n]) { *end = s; *steps = k; return 1; }
    }
    return 0;
}

/* ------------------------------- MemImage -------------------------------- */

uint64_t or_memimage_get(const uint64_t* data, uint32_t state_len, uint64_t i) {
    const uint32_t w = state_len + 1;
    const uint64_t mask = w >= 64 ? ~0ull : ((1ull << w) - 1);
    uint64_t bitpos = i * w;
    uint64_t idx = bitpos >> 6, bit = bitpos & 63;
    if (64 - bit >= w) return (data[idx] >> bit) & mask;
    return ((data[idx] >> bit) | (data[idx + 1] << (64 - bit))) & mask;
}

void or_memimage_set(uint64_t* data, uint32_t state_len, uint64_t i, uint64_t value) {
    const uint32_t w = state_len + 1;
    const uint64_t mask = w >= 64 ? ~0ull : ((1ull << w) - 1);
    value &= mask;
    uint64_t bitpos = i * w;
    uint64_t idx = bitpos >> 6, bit = bitpos & 63;
    data[idx] = (data[idx] & ~(mask << bit)) | (value << bit);
    if (64 - bit < w)
        data[idx + 1] = (data[idx + 1] & ~(mask >> (64 - bit))) | (value >> (64 - bit));
}

int or_memimage_find_solution(const uint64_t* data, uint32_t state_len,
                              uint64_t start, uint64_t len, uint32_t unknowns,
                              uint64_t* sol_start, uint64_t* sol_end) {
    if (unknowns > state_len) return -1;
    const uint64_t before = (1ull << (state_len - unknowns)) - 1;
    const uint64_t stepv = before + 1;
    uint64_t us = (start & before) ? (start & ~before) + stepv : (start & ~before);
    const uint64_t endv = start + len;
    const uint64_t smask = (1ull << state_len) - 1;
    const uint64_t stopbit = 1ull << state_len;
    for (uint64_t s = us; s < endv; s += stepv) {
        uint64_t v = or_memimage_get(data, state_len, s - start);
        if (v & stopbit) { *sol_start = s; *sol_end = v & smask; return 1; }
    }
    return 0;
}

/* MemImage::join_nexts (greedysatostop.rs:433-481) on packed partitions of
 * len entries; second covers states [start2, start2 + len). */
static void or_join_nexts(uint64_t* dest, const uint64_t* second, uint32_t n, uint64_t len, uint64_t start2) {
    const uint64_t smask = (1ull << n) - 1, stopbit = 1ull << n;
    for (uint64_t i = 0; i < len; i++) {
        const uint64_t v = or_memimage_get(dest, n, i);
        const uint64_t nx = v & smask;
        if (!(v & stopbit) && nx >= start2 && nx < start2 + len)
            or_memimage_set(dest, n, i, or_memimage_get(second, n, nx - start2));
    }
}

int or_greedy_partitioned(const uint64_t* table, uint32_t n, uint32_t unknowns, uint32_t partitions,
                          uint64_t* start, uint64_t* end, uint32_t* stage, uint32_t* part) {
    if (n < 6 || n > 40 || unknowns > n || partitions < 2 || (partitions & (partitions - 1)) ||
        (uint64_t)partitions * 64 > (1ull << n))
        return -1;
    const uint64_t N = 1ull << n, L = N / partitions;
    const uint64_t pwords = (L * (n + 1)) >> 6;
    uint64_t* image = (uint64_t*)calloc((N * (n + 1)) >> 6, 8);
    uint64_t* dest = (uint64_t*)calloc(pwords, 8);
    uint64_t* second = (uint64_t*)calloc(pwords, 8);
    if (!image || !dest || !second) { free(image); free(dest); free(second); return -1; }
    int have_stop = 0;
    for (uint64_t s = 0; s < N; s++) {
        or_memimage_set(image, n, s, table[s]);
        have_stop |= (table[s] >> n) & 1;
    }
    int found = 0;
    for (uint32_t st = 0; have_stop && st < n && !found; st++) {
        for (uint32_t i = 0; i < partitions && !found; i++) {
            memcpy(dest, image + i * pwords, pwords * 8);
            for (uint32_t j = 0; j < partitions; j++) {
                if (j != i) memcpy(second, image + j * pwords, pwords * 8);
                else memcpy(second, dest, pwords * 8);
                or_join_nexts(dest, second, n, L, (uint64_t)j * L);
            }
            if (or_memimage_find_solution(dest, n, (uint64_t)i * L, L, unknowns, start, end) == 1) {
                *stage = st;
                *part = i;
                found = 1;
            } else {
                memcpy(image + i * pwords, dest, pwords * 8);
            }
        }
    }
    free(image); free(dest); free(second);
    return found;
}

/*
 * nsat_oracle.h -- CPU restatement of the reference solvers' semantics.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker that the CUDA path is
 * compared against, and the timed CPU baseline ("port") of the reference's
 * gatenative CPU path.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it.  The product (libnsat) never links or calls it.
 *
 * Circuit encoding (shared with the product C ABI, include/nsat.h):
 *   wires 0..n-1 are circuit inputs, wire n+k is gate k;
 *   gates[3k+0] = function (0=AND, 1=NOR, 2=NIMPL, 3=XOR), gates[3k+1] = i0,
 *   gates[3k+2] = i1 (both < n+k);
 *   outputs[2j+0] = wire, outputs[2j+1] = negated flag.
 * Gate meaning follows gatesim's GateFunc (And: i0&i1, Nor: !(i0|i1),
 * Nimpl: i0&!i1, Xor: i0^i1) as used by Circuit::new(n, gates, outputs)
 * at qsat.rs:2630 and satostop.rs:1792 of the reference.
 */
#ifndef NSAT_ORACLE_H
#define NSAT_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct {
    uint32_t n;               /* input count */
    uint32_t g;               /* gate count */
    const uint32_t* gates;    /* 3*g */
    uint32_t o;               /* output count */
    const uint32_t* outputs;  /* 2*o */
} or_circuit;

/* Scalar evaluation: in[i] in {0,1} for every input, out[j] in {0,1}. */
int or_eval_scalar(const or_circuit* c, const uint8_t* in, uint8_t* out);

/* Bit-sliced evaluation of 64 assignments: in[i] is a 64-lane word for
 * input i, out[j] receives the 64-lane word of output j. */
int or_eval_words(const or_circuit* c, const uint64_t* in, uint64_t* out);

/* SAT over natural order (input b = bit b of the index), main.rs:76-155,
 * 266-382.  Scans indices [begin, end) (end <= 2^n, n <= 63); returns the
 * exact solution count and the lowest satisfying index (UINT64_MAX if none).
 * threads <= 0 means all OpenMP threads. */
int or_sat_range(const or_circuit* c, uint64_t begin, uint64_t end, int threads,
                 uint64_t* count, uint64_t* lowest);

/* ---- QuantReducer (qsat.rs:172-291) ------------------------------------ */
typedef struct or_qr or_qr;
/* quants[i]: 1 = All (forall), 0 = Exists, for input i; nq <= 64 */
or_qr* or_qr_new(const uint8_t* quants, int nq);
void or_qr_free(or_qr* qr);
int or_qr_push(or_qr* qr, uint64_t index, int item);
/* pushes item k = bit k%32 of words[k/32] for k = 0.. in order, until final */
int or_qr_push_words(or_qr* qr, const uint32_t* words, uint64_t nwords);
int or_qr_push_words_from(or_qr* qr, uint64_t first, const uint32_t* words, uint64_t nwords);
/* returns 1 and fills the FinalResult fields when final, else 0 */
int or_qr_final(const or_qr* qr, int* reversed, uint32_t* solution_bits,
                int* has_solution, uint64_t* solution);

/* Full QSAT in v-order (input i = bit n-1-i of v), qsat.rs:1991-1998:
 * the answer of pushing every circuit value, in order, into a QuantReducer.
 * mode 0: one QuantReducer over all 2^n items (single thread, small n);
 * mode 1: OpenMP chunks on the top bits joined by a top QuantReducer,
 *         the arrangement of MainCPUQuantReducer (qsat.rs:1327-1397). */
int or_qsat(const or_circuit* c, const uint8_t* quants, int mode, int threads,
            int* reversed, uint32_t* solution_bits, int* has_solution,
            uint64_t* solution);

/* ---- SATOSTOP (greedysatostop.rs:142-302, 634-690; satostop.rs:1751) ---- */
/* Next-state table: table[s] = next(s) | STOP(s) << n, input b = bit b of s.
 * Circuit must have n inputs and n+1 outputs; n <= 32 here. */
int or_stop_table(const or_circuit* c, int threads, uint64_t* table);

/* Synchronous pointer doubling over the table (rounds of
 * T'[s] = STOP(T[s]) ? T[s] : T[next(T[s])], at most n rounds), after the
 * check_stop of greedysatostop.rs:196-236.  Starts are the states whose low
 * n-u bits are zero.  mode 0: return the lowest start resolved in the first
 * round that resolves any start (greedysatostop's loop, 662-686);
 * mode 1: the lowest start that stops at all (naivesatostop -S order).
 * steps = evaluations from start to the stopping evaluation, inclusive. */
int or_stop_solve(uint32_t n, uint32_t u, const uint64_t* table, int mode,
                  int threads, int* found, uint64_t* start, uint64_t* end,
                  uint64_t* steps, uint32_t* rounds);

/* Replay from start until STOP (greedysatostop.rs:1114-1134,
 * satostop.rs:1723-1745); stops after max_steps evaluations.
 * Returns 1 if stopped (end/steps filled), 0 otherwise. */
int or_stop_replay(const or_circuit* c, uint64_t start, uint64_t max_steps,
                   uint64_t* end, uint64_t* steps);

/* ---- MemImage packed (n+1)-bit entries (greedysatostop.rs:308-489) ----- */
uint64_t or_memimage_get(const uint64_t* data, uint32_t state_len, uint64_t i);
void or_memimage_set(uint64_t* data, uint32_t state_len, uint64_t i, uint64_t value);
/* find_solution on an image of len entries starting at state `start` */
int or_memimage_find_solution(const uint64_t* data, uint32_t state_len,
                              uint64_t start, uint64_t len, uint32_t unknowns,
                              uint64_t* sol_start, uint64_t* sol_end);

/* Partitioned greedysatostop (greedysatostop.rs:692-837,
 * do_solve_with_cpu_builder_with_partitions) on a packed MemImage of the
 * table T[s] = next | STOP << n: for stage 0..n-1 and partition i, dest =
 * partition i joined with every partition j in order (the image's current
 * copy, or dest itself for j == i, greedysatostop.rs:796-806), then
 * find_solution on dest, else dest is written back.  Returns 1 with the
 * answer and where it was found, 0 if none, -1 on bad arguments. */
int or_greedy_partitioned(const uint64_t* table, uint32_t n, uint32_t unknowns, uint32_t partitions,
                          uint64_t* start, uint64_t* end, uint32_t* stage, uint32_t* part);

#ifdef __cplusplus
}
#endif
#endif

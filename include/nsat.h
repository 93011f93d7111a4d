/*
 * nsat.h -- C ABI of the B200 exhaustive circuit solver (libnsat.so).
 *
 * The reference (matszpk/naivesat) plugs its solvers into the external
 * gatenative crate: a builder compiles a Gate circuit plus a C/OpenCL
 * "aggr_output" snippet into a bit-sliced kernel, and a mapper calls it once
 * per value of the "arg" inputs (main.rs:106-264, qsat.rs:1599-1836,
 * greedysatostop.rs:634-837, 1042-1099).  This ABI replaces that whole
 * builder/mapper/snippet stack with one call per solve.  Every entry point
 * returns an int status (0 = OK, negative = error, never aborts); a context is
 * bound to one device and one stream and must not be used by two threads at
 * once; separate contexts are independent.
 *
 * Circuit encoding: wires 0..n-1 are the inputs, wire n+k is gate k.
 *   gates[3k] = function (NSAT_AND/NOR/NIMPL/XOR), gates[3k+1] = i0,
 *   gates[3k+2] = i1 (< n+k);  outputs[2j] = wire, outputs[2j+1] = negated.
 * This is the shape of gatesim's Circuit::new(n, gates, outputs) as used at
 * qsat.rs:2630 and satostop.rs:1792.
 */
#ifndef NSAT_H
#define NSAT_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define NSAT_OK 0
#define NSAT_EINVAL (-1)        /* bad argument or malformed circuit */
#define NSAT_ENOMEM (-2)        /* host or device allocation failed */
#define NSAT_ECOMPILE (-3)      /* NVRTC compile or module load failed */
#define NSAT_ECUDA (-4)         /* a CUDA call failed */
#define NSAT_ETIMEOUT (-5)      /* a bounded device wait ran out */
#define NSAT_ENODEV (-6)        /* no usable CUDA device */
#define NSAT_EUNSUPPORTED (-7)  /* size outside what this build handles */
#define NSAT_EPARSE (-8)        /* circuit text could not be parsed */
#define NSAT_EBUSY (-9)         /* admission refused (serving queue full) */

enum { NSAT_AND = 0, NSAT_NOR = 1, NSAT_NIMPL = 2, NSAT_XOR = 3 };

typedef struct nsat_ctx nsat_ctx;
typedef struct nsat_circuit nsat_circuit;
typedef struct nsat_table nsat_table;
typedef struct nsat_parsed nsat_parsed;

typedef struct {
    uint32_t input_len;
    uint32_t gate_num;
    const uint32_t* gates;    /* 3 * gate_num */
    uint32_t output_num;
    const uint32_t* outputs;  /* 2 * output_num */
} nsat_circuit_desc;

typedef struct {
    uint32_t block_threads;   /* CUDA block size; 0 = auto.  The reference's -G
                                 (OpenCL group length, main.rs:70-73) maps here */
    uint32_t no_optimize;     /* 1 = one logic op per gate, no LOP3 cut mapping.
                                 The reference's -n (optimize_negs off) maps here */
    uint32_t verbose;         /* 1 = print JIT/launch details on stderr */
    uint32_t min_blocks;      /* CTAs per SM the kernels are compiled for
                                 (__launch_bounds__ minimum); 0 = auto */
} nsat_opts;

/* ---- context ------------------------------------------------------------ */
/* Replaces OpenCLBuilder::new(&device, config) / CPUBuilder::new (main.rs:278-300).
 * A context owns a stream and a stream-ordered device memory pool for per-call
 * buffers (SATOSTOP tables, partitioned images): freed buffers stay in the
 * pool for the next call, up to 8 GiB; nsat_destroy returns them.  Tables are
 * freed (nsat_table_free) before their context. */
int nsat_create(int device, const nsat_opts* opts, nsat_ctx** out);
void nsat_destroy(nsat_ctx* ctx);
const char* nsat_strerror(int status);
/* Last error detail of this context (empty string if none). */
const char* nsat_last_error(const nsat_ctx* ctx);
/* Number of visible CUDA devices (0 when none); never fails. */
int nsat_device_count(void);

/* ---- circuits ----------------------------------------------------------- */
/* Replaces builder.add_with_config(name, circuit, CodeConfig) (main.rs:113-123):
 * validates and copies the circuit; kernels are generated and NVRTC-compiled
 * lazily on first use per solve kind and cached by content hash. */
int nsat_circuit_new(nsat_ctx* ctx, const nsat_circuit_desc* desc, nsat_circuit** out);
/* Frees the handle and the kernels only it still holds (on its device; the
 * caller's current device is restored).  Free circuits before their context. */
void nsat_circuit_free(nsat_circuit* c);
/* LUT statistics after cut mapping of output `output` (or all outputs when
 * output < 0): live two-input gates and LOP3 operations emitted. */
int nsat_circuit_stats(nsat_ctx* ctx, nsat_circuit* c, int output,
                       uint32_t* live_gates, uint32_t* lop3_ops);

/* Parses gatesim text: Circuit::from_str (main.rs:390) or, with a quantifier
 * prefix, QuantCircuit::from_str (qsat.rs:6276-6285). */
int nsat_parse(const char* text, size_t len, nsat_parsed** out);
/* quants: NULL if the text had no quantifiers, else input_len bytes, 1 = All. */
int nsat_parsed_get(const nsat_parsed* p, nsat_circuit_desc* desc, const uint8_t** quants);
void nsat_parsed_free(nsat_parsed* p);
/* Writes gatesim text; returns the needed size (without NUL) in *needed. */
int nsat_format(const nsat_circuit_desc* desc, const uint8_t* quants, char* buf,
                size_t buflen, size_t* needed);

/* ---- SAT (naivesat) ----------------------------------------------------- */
/* Replaces do_command_with_{par,opencl,parseq}_mapper with AGGR_OUTPUT_*_CODE
 * (main.rs:76-264).  Natural order: input b is bit b of the assignment index.
 * Output 0 of the circuit is the formula. */
/* A chunk queue shared by several concurrent solves of one SAT search, one
 * context per device, each on its own host thread: the counterpart of the
 * reference's ParSeq mapper, which hands args to whichever device is free and
 * stops every device once one holds a witness (main.rs:205-264).
 * Zero-initialise one, then give the same object, range and chunk_bits to
 * every participant's nsat_sat_solve (find_all = 0).  Participants claim
 * chunks (launches) in increasing order with an atomic counter; a chunk
 * holding a solution lowers `stop_plus1`, and nobody claims a chunk at or
 * above it.  Every chunk below the final stop is evaluated by some
 * participant, so the lowest of their witnesses is the range's lowest.
 * Accessed with host atomics only; it must outlive the solves. */
typedef struct {
    uint64_t next;         /* next chunk to claim, counted from the range's start */
    uint64_t stop_plus1;   /* 0, or 1 + the lowest chunk known to hold a solution */
    uint64_t reserved[6];
} nsat_sat_share;

typedef struct {
    uint32_t find_all;     /* 0: stop after the first chunk holding a solution and
                              return the lowest one (naivesat); 1: scan the
                              whole range, exact count and lowest witness */
    uint32_t chunk_bits;   /* log2 assignments per launch (0 = auto).  The
                              reference's -e elem_inputs maps here */
    uint64_t begin_lo, begin_hi;  /* first index of the range (chunk aligned) */
    uint64_t end_lo, end_hi;      /* end of range; both 0 = 2^n */
    nsat_sat_share* share;        /* NULL, or the queue of a search split over
                                     several contexts (find_all must be 0); the
                                     result then covers this context's chunks */
} nsat_sat_opts;

typedef struct {
    int32_t satisfiable;
    uint32_t launches;
    uint64_t count_lo, count_hi;      /* solutions among the scanned indices */
    uint64_t witness_lo, witness_hi;  /* lowest satisfying index */
    uint64_t scanned_lo, scanned_hi;  /* assignments scanned */
    double device_ms;                 /* kernel time, CUDA events */
    double wall_ms;                   /* host time of the call */
} nsat_sat_result;

int nsat_sat_solve(nsat_ctx* ctx, nsat_circuit* c, const nsat_sat_opts* opts,
                   nsat_sat_result* res);

/* ---- QSAT (naiveqsat) --------------------------------------------------- */
/* Replaces MainOpenCLQuantReducer/OpenCLQuantReducer/QuantReducer and the
 * QSAT aggr snippets (qsat.rs:172-1597).  v-order: input i is bit n-1-i of
 * the item index, so input 0 is the outermost quantifier.  The answer equals
 * pushing every circuit value in order into a QuantReducer (qsat.rs:1991). */
typedef struct {
    uint32_t chunk_bits;   /* log2 assignments per launch (0 = auto) */
    uint32_t prefix_bits;  /* fix inputs 0..prefix_bits-1 (the outermost
                              quantifiers) to `prefix` and solve the formula
                              below them: the result then describes the
                              sub-formula over inputs prefix_bits..n-1 (its
                              first block, its value).  Shards of a multi-GPU
                              solve use this; 0 = the whole formula */
    uint64_t prefix;       /* input 0 is the most significant of prefix_bits */
} nsat_qsat_opts;

typedef struct {
    int32_t reversed;          /* first quantifier is All */
    uint32_t solution_bits;    /* length of the first quantifier block */
    int32_t has_solution;
    int32_t value;             /* truth value of the quantified formula */
    uint64_t solution_lo, solution_hi;  /* bit k = input k of the first block */
    uint32_t launches;
    uint32_t chunk_bits;       /* log2 assignments per launch actually used */
    uint64_t scanned;          /* assignments evaluated (launches x 2^chunk_bits) */
    double device_ms;
    double wall_ms;
} nsat_qsat_result;

int nsat_qsat_solve(nsat_ctx* ctx, nsat_circuit* c, const uint8_t* quants,
                    const nsat_qsat_opts* opts, nsat_qsat_result* res);

/* nsat_qsat_solve for callers that cannot call cudaMalloc -- for example a
 * serving process whose device memory belongs to another allocator or a fixed
 * budget, where cudaMalloc/cudaFree would synchronize the device or break the
 * budget mid-request.  No counterpart in the reference (its OpenCL reducer
 * allocates its buffers per solver, qsat.rs:1046-1064).
 * The last-CTA scratch comes from a static device array of
 * NSAT_NOALLOC_SCRATCH_BYTES (64 KiB) inside libnsat.so instead of the
 * context's lazily allocated buffer; every GPU that loads the library holds it
 * until exit.  A solve whose launches need more scratch (2 << CB bytes, CB =
 * log2 CTAs per launch, so launches of up to 2^15 CTAs fit) fails with
 * NSAT_EUNSUPPORTED before any kernel is compiled; lower chunk_bits then.
 * The first call on a device looks the array up (cudaGetSymbolAddress) and the
 * first call for a circuit/quantifier string compiles and loads its kernel;
 * make that first call before any stream capture.  All calls share the one
 * array: calls that overlap on the GPU (several contexts on one device, or
 * other threads) race on it and must be serialised by the caller.  Results
 * equal nsat_qsat_solve's. */
#define NSAT_NOALLOC_SCRATCH_BYTES (64u * 1024u)
int nsat_qsat_solve_noalloc(nsat_ctx* ctx, nsat_circuit* c, const uint8_t* quants,
                            const nsat_qsat_opts* opts, nsat_qsat_result* res);

/* Runs the QSAT reduction kernel on raw item bits instead of a circuit
 * (item k = bit k%32 of words[k/32], 2^nq items, nq >= 5): the analogue of
 * the reference's identity-circuit aggregator tests (qsat.rs:2629-3520). */
int nsat_qsat_reduce_words(nsat_ctx* ctx, const uint8_t* quants, uint32_t nq,
                           const uint32_t* words, nsat_qsat_result* res);

/* ---- SATOSTOP (greedysatostop, naivesatostop) ---------------------------- */
/* Replaces the greedy OpenCL table aggr + join_nexts/check_stop/find_solution
 * kernels (greedysatostop.rs:841-1099).  The circuit has n inputs and n+1
 * outputs: outputs 0..n-1 are the next state, output n is STOP. */
typedef struct {
    uint32_t want_steps;   /* carry evaluation counts (naivesatostop's steps) */
    uint32_t reserved;
} nsat_table_opts;

int nsat_stop_table_build(nsat_ctx* ctx, nsat_circuit* c, const nsat_table_opts* opts,
                          nsat_table** out);
void nsat_table_free(nsat_table* t);
/* Copies entries [first, first+count) as next | STOP << n (device -> host). */
int nsat_table_read(nsat_table* t, uint64_t first, uint64_t count, uint64_t* out);
/* Bytes of device memory held by the table (both ping-pong buffers). */
uint64_t nsat_table_bytes(const nsat_table* t);

typedef struct {
    uint32_t unknowns;     /* the top `unknowns` state bits are the unknowns */
    uint32_t mode;         /* 0: lowest start among those resolved in the first
                              doubling round that resolves any (greedy loop,
                              greedysatostop.rs:1084-1091); 1: lowest start
                              that stops at all (naivesatostop -S order) */
} nsat_stop_opts;

typedef struct {
    int32_t found;
    uint32_t rounds;       /* doubling rounds run */
    uint64_t start, end, steps;   /* steps only with want_steps */
    double build_ms, join_ms;
} nsat_stop_result;

int nsat_stop_solve(nsat_ctx* ctx, nsat_table* t, const nsat_stop_opts* opts,
                    nsat_stop_result* res);

/* ---- autotuning ----------------------------------------------------------
 * Times the evaluator kernels of one circuit over a sample of its index
 * space with candidate launch shapes -- threads per CTA, CTAs per SM the
 * kernels are compiled for (the register budget), CTA bits per launch
 * against loop iterations per warp, and the spacing of CTA barriers that keep
 * a CTA's warps on the same instruction-cache lines -- and keeps the fastest on the circuit
 * handle: later nsat_sat_solve / nsat_qsat_solve calls on that handle use it.
 * Answers are the same under every shape.  Candidates are compiled in
 * parallel host threads.  With persist the choice is reused from / stored in
 * the kernel cache directory, keyed by circuit, kind, quantifiers and GPU.
 * No counterpart in the reference (its OpenCL group length is a flag). */
typedef struct {
    uint32_t kind;            /* 0 SAT, 1 QSAT */
    uint32_t persist;         /* 1: reuse / store the choice in the kernel cache directory */
    const uint8_t* quants;    /* QSAT: one per input, 1 = All */
    double sample_ms;         /* device time measured per candidate (0 = 60 ms) */
    uint32_t threads;         /* host compile threads (0 = hardware threads) */
    uint32_t reserved;
} nsat_tune_opts;

typedef struct {
    uint32_t block_threads, min_blocks, cta_bits_max;   /* the chosen shape */
    uint32_t candidates;      /* shapes timed (0 when taken from the cache) */
    uint32_t from_cache;
    uint32_t sync_every;      /* CTA barrier every this many LUTs in the evaluation (0 = none) */
    double best_rate;         /* assignments per second with the chosen shape */
    double default_rate;      /* ... with the context's shape */
    double tune_ms;           /* wall time of tuning */
} nsat_tune_result;

int nsat_autotune(nsat_ctx* ctx, nsat_circuit* c, const nsat_tune_opts* opts, nsat_tune_result* res);
/* Forgets a circuit's tuned shapes: its solves use the context's options. */
int nsat_autotune_reset(nsat_circuit* c);

/* ---- partitioned greedysatostop (greedysatostop -p P [-x PREFIX]) -------
 * Replaces do_solve_with_cpu_builder_with_partitions
 * (greedysatostop.rs:692-837): the table is kept as a packed image of
 * (n+1)-bit entries (MemImage/FileImage layout, greedysatostop.rs:308-594)
 * and joined partition by partition in the reference's order, so the answer
 * is the reference's for every P.  The image lives in device memory when it
 * fits, else in pinned host memory (partitions cross PCIe, double-buffered),
 * or with file_prefix in the temp file <file_prefix>greedy_temp_<ns>
 * (deleted before return).  Work buffers: two unpacked partitions
 * (2^(n - log2 P) x 8 bytes each), plus staging for a host or file image. */
typedef struct {
    uint32_t unknowns;
    uint32_t partitions;        /* power of two >= 2, partitions * 64 <= 2^n */
    const char* file_prefix;    /* image in a temp file under this prefix (greedysatostop -x) */
    uint64_t device_bytes;      /* without a file: the image stays in device memory when it and the
                                   work buffers fit in this many bytes (0 = free device memory less
                                   1 GiB), else it spills to pinned host memory */
} nsat_greedy_opts;

typedef struct {
    int32_t found;
    uint32_t stage, partition;  /* where the answer was found */
    uint32_t load_bits;         /* first-pass chunks: 2^load_bits ("Load partition bits") */
    uint32_t storage;           /* where the image lived: 0 device memory, 1 pinned host memory, 2 file */
    uint32_t reserved;
    uint64_t start, end;
    uint64_t joins;             /* partition joins run */
    double build_ms, join_ms, wall_ms;   /* table kernels, join kernels (CUDA events); wall */
    uint64_t h2d_bytes, d2h_bytes;       /* image traffic over PCIe */
} nsat_greedy_result;

int nsat_greedy_solve(nsat_ctx* ctx, nsat_circuit* c, const nsat_greedy_opts* opts, nsat_greedy_result* res);
/* The packed image after the first pass (ceil(2^n (n+1) / 64) words), for
 * checking the layout; the partition count sets the first pass's chunking. */
int nsat_greedy_image(nsat_ctx* ctx, nsat_circuit* c, uint32_t partitions, const char* file_prefix,
                      uint64_t* words, uint64_t nwords);

/* ---- batched serving ---------------------------------------------------- */
/* A server runs many SAT / QSAT / SATOSTOP jobs on one device concurrently
 * (no counterpart in the reference, which solves one circuit per process).
 * Circuits are interpreted as LUT bytecode by one precompiled kernel, so a
 * new circuit costs no compilation; jobs are admitted in arrival order while
 * their device memory fits the server's budget; every nsat_server_step runs
 * one epoch (one CUDA-graph replay) over a slice of tiles (2^15 assignments)
 * of every active job, slices doubling from one tile, and retires finished
 * jobs.  Answers equal the one-shot solvers': SAT the lowest witness, QSAT
 * the QuantReducer result, SATOSTOP the lowest stopping start with steps. */
typedef struct nsat_server nsat_server;

typedef struct {
    uint64_t arena_bytes;       /* device memory for admitted jobs; 0 = 1 GiB */
    uint32_t max_active;        /* jobs sharing the device at once (<= 512); 0 = 512 */
    uint32_t max_queue;         /* waiting jobs before submit returns NSAT_EBUSY; 0 = 2^20 */
    uint32_t max_slice_tiles;   /* cap of one job's tiles per epoch; 0 = 4096 */
    uint32_t first_slice_tiles; /* a new job's first slice (doubling after); 0 = 256 */
    uint64_t epoch_budget;      /* sum over jobs of tiles x program length per epoch; 0 = the
                                   budget nsat_server_tune persisted for this GPU, else 1.2e7
                                   (on a mixed serving trace: the most solves/s, the same p99
                                   as 6e6-4.8e7) */
    uint32_t build_threads;     /* host threads that build job programs; 0 = min(8, cores / 2) */
    uint32_t tier_threads;      /* QSAT tiering workers (own context each); 0 = three quarters of
                                   the host threads, between 2 and 12 */
    uint32_t tier_min_ms;       /* QSAT jobs whose whole index space would take the interpreter
                                   longer than this (estimate) race a compiled kernel: it is
                                   compiled in the background and, once ready, solves the job's
                                   remaining 1/16 blocks as prefix sub-problems; 0 = 30,
                                   0xFFFFFFFF = never */
    uint32_t tier_wait;         /* 1: such a job is not interpreted until its kernel is ready, so
                                   every block runs compiled (compile first instead of racing) */
    uint32_t shape;             /* interpreter shape, 1..NSAT_SERVE_SHAPES (below); 0 = the shape
                                   nsat_server_tune persisted for this GPU, else the default */
    uint32_t rollover;          /* 1: warps that run out of planned work go on into the next
                                   quarter slice of undecided SAT and SATOSTOP jobs, with no host
                                   round trip; 0: each epoch evaluates exactly its slices */
} nsat_server_opts;

/* Interpreter shapes: words per lane W (W x 1024 assignments per warp and
 * program pass), groups of G mutually independent instructions (a group's
 * operands are loaded before any result is stored), and the evaluation of a
 * LUT with a run-time truth table, either a 7-lop3 mux tree over masks or a
 * jump on the warp-uniform table to one lop3 per word:
 *   1: W4 G4 mux   2: W4 G1 jump   3: W4 G2 jump
 *   4: W4 G4 jump  5: W2 G1 jump   6: W2 G2 jump */
#define NSAT_SERVE_SHAPES 6

typedef struct {
    uint32_t kind;              /* 0 = SAT, 1 = QSAT, 2 = SATOSTOP */
    uint32_t unknowns;          /* SATOSTOP: the top `unknowns` state bits */
    const uint8_t* quants;      /* QSAT: one per input, 1 = All */
    nsat_circuit_desc circuit;
    uint64_t tag;               /* returned with the result */
    uint32_t flags;             /* NSAT_JOB_FIND_ALL: a SAT job counts every solution */
    uint32_t reserved;
} nsat_job_desc;

#define NSAT_JOB_FIND_ALL 1u

typedef struct {
    uint64_t id, tag;
    int32_t status;
    uint32_t kind;
    int32_t satisfiable;        /* SAT */
    int32_t value;              /* QSAT: truth value */
    uint64_t witness_lo, witness_hi;   /* SAT: lowest satisfying index */
    uint64_t count;             /* SAT: solutions in the evaluated tiles */
    int32_t reversed;           /* QSAT FinalResult */
    uint32_t solution_bits;
    int32_t has_solution;
    int32_t found;              /* SATOSTOP */
    uint64_t solution;
    uint64_t start, end, steps; /* SATOSTOP */
    uint64_t tiles;             /* tiles evaluated by the interpreter */
    double submit_ms, admit_ms, done_ms;   /* steady clock, milliseconds */
    uint32_t compiled_blocks;   /* QSAT: prefix blocks solved by a compiled kernel (tiering) */
    uint32_t epochs;            /* epochs that evaluated a slice of this job */
    uint64_t first_epoch;       /* sequence number (from 1) of the first epoch that ran a slice of
                                   this job, and of the last one; 0 when no epoch ran it.  Jobs
                                   whose [first_epoch, last_epoch] ranges intersect shared the
                                   device in those epochs. */
    uint64_t last_epoch;
} nsat_job_result;

typedef struct {
    uint64_t epochs;
    double device_ms;           /* interpreter kernel time, CUDA events */
    uint32_t active, queued;
    uint64_t arena_used, arena_bytes;
    uint32_t graph_slots, grid;
    uint64_t launches;          /* kernels launched: epoch graphs and join rounds */
    uint64_t h2d_bytes, d2h_bytes;   /* host<->device copies issued: programs, epoch tables, results */
    uint32_t shape;             /* the interpreter shape in use (1-based) */
    uint32_t reserved;
} nsat_server_stats_t;

/* Autotuner of the batched interpreter (no counterpart in the reference).
 * Serves a seeded calibration set of SAT jobs in count mode (every tile
 * evaluated, so the work is fixed: 24-30 inputs, 100-4000 gates) under every
 * interpreter shape and keeps the one with the most LUT-words per second of
 * device time; then, for that shape, times the same set with epoch budgets of
 * 1.2e7 .. 9.6e7.  The set measures throughput, not the latency of arrivals,
 * so the default budget (1.2e7) stays unless another is more than 5 % faster
 * with a mean epoch under 20 ms.  With `persist` the
 * choice is written to the kernel cache directory, keyed by GPU, and servers
 * created later with shape 0 and epoch_budget 0 use it; an existing choice is
 * read back instead of timing again unless `retune` is set. */
typedef struct {
    uint32_t jobs;          /* calibration jobs (0 = 24) */
    uint32_t persist;
    uint32_t retune;        /* time again even if a persisted choice exists */
    uint32_t reserved;
    uint64_t seed;          /* calibration set (0 = the fixed default) */
} nsat_serve_tune_opts;

typedef struct {
    uint32_t shape;                                /* chosen, 1-based */
    uint32_t from_cache;                           /* read back, nothing timed */
    uint64_t epoch_budget;                         /* chosen */
    double lut_words_per_s[NSAT_SERVE_SHAPES];     /* per shape, device time (0 = not timed) */
    double budget_solves_per_s[4];                 /* budgets 6e6, 1.2e7, 2.4e7, 4.8e7: wall clock */
    double budget_epoch_ms[4];                     /* their mean epoch wall time */
    double tune_ms;
} nsat_serve_tune_result;

int nsat_server_tune(nsat_ctx* ctx, const nsat_serve_tune_opts* opts, nsat_serve_tune_result* res);

int nsat_server_create(nsat_ctx* ctx, const nsat_server_opts* opts, nsat_server** out);
void nsat_server_destroy(nsat_server* s);
/* Queues a job (the circuit is copied) and returns at once: its program is
 * built on the server's builder threads.  NSAT_EBUSY when the queue is full;
 * malformed jobs are refused here.  A job whose program cannot be served
 * (more slots than the interpreter holds: NSAT_EUNSUPPORTED; larger than the
 * arena: NSAT_ENOMEM) comes back from nsat_server_poll with that status.
 * submit, step and poll are meant for one caller thread. */
int nsat_server_submit(nsat_server* s, const nsat_job_desc* job, uint64_t* id);
/* Admits what fits and runs one epoch; reports jobs still active / queued. */
int nsat_server_step(nsat_server* s, uint32_t* active, uint32_t* queued);
/* Moves up to `cap` finished results to `out`. */
int nsat_server_poll(nsat_server* s, nsat_job_result* out, uint32_t cap, uint32_t* n);
int nsat_server_stats(nsat_server* s, nsat_server_stats_t* st);

/* Host-only check of the interpreter program a job of `kind` would get on a
 * server of `shape` (1-based; 0 = the default shape): builds it, runs it on
 * the host with the kernel's group semantics (a group's operands are read
 * before any of its results is written) for two passes of 64 seeded random
 * assignments, and compares every requested output with direct evaluation
 * of the circuit.  Reports the program's slots, LUTs and padding NOPs.
 * NSAT_EINVAL on a mismatch.  Needs no GPU. */
int nsat_server_program_check(const nsat_circuit_desc* circuit, uint32_t kind, uint32_t shape, uint64_t seed,
                              uint32_t* slots, uint32_t* luts, uint32_t* nops);

/* ---- seeded benchmark circuits ------------------------------------------- */
/* Random DAG of the benchmark configurations: `gates` two-input gates, types
 * uniform over the four, each fan-in uniform over the preceding `window`
 * wires and negated with probability 1/4 (negations folded into the gate
 * functions); the single output is the last gate, or with live_output the last
 * gate that is not constant on 4096 seeded samples.  splitmix64(seed) drives
 * every draw.  Writes up to gate_cap gates / out_cap outputs; returns the
 * counts. */
int nsat_gen_random_dag(uint64_t seed, uint32_t n, uint32_t gates, uint32_t window, int live_output,
                        uint32_t* out_gates, uint32_t gate_cap, uint32_t* out_outputs, uint32_t out_cap,
                        uint32_t* gate_num, uint32_t* out_num);
/* SATOSTOP next-state circuit: n-bit Fibonacci LFSR (4 seeded taps, n-1
 * among them) XOR the last n gates of a seeded `mixer_gates`-gate random DAG;
 * STOP = (state == seeded pattern).  n+1 outputs. */
int nsat_gen_lfsr_stop(uint64_t seed, uint32_t n, uint32_t mixer_gates, uint32_t* out_gates,
                       uint32_t gate_cap, uint32_t* out_outputs, uint32_t out_cap, uint32_t* gate_num,
                       uint32_t* out_num, uint64_t* pattern);

/* ---- build check -------------------------------------------------------- */
/* Generates and NVRTC-compiles for sm_100a, without a device, the kernel that
 * a solve of `kind` (0 = SAT, 1 = QSAT, 2 = SATOSTOP table) would launch for
 * this circuit, and reports ptxas resource usage.  Plays the role of the
 * reference's mapper.build() step (main.rs:124), minus the device.
 * quants is required for kind 1.  log (may be NULL) receives the compile log. */
typedef struct {
    int32_t regs;           /* registers per thread */
    int32_t spill_bytes;    /* spill stores per thread */
    uint32_t lop3_ops;      /* LOP3 operations per 32-lane word */
    uint32_t live_gates;    /* two-input gates in the output cone */
    double compile_ms;
} nsat_jit_info;

int nsat_jit_check(const nsat_circuit_desc* desc, const uint8_t* quants, int kind,
                   const nsat_opts* opts, nsat_jit_info* info, char* log, size_t loglen);

/* ---- measurement -------------------------------------------------------- */
/* Measures this device's 32-bit LOP3 issue rate with a chain microbenchmark
 * (independent lop3.b32 chains, no memory traffic): thread-instructions/s. */
int nsat_probe_lop3_peak(nsat_ctx* ctx, double* lop3_per_s, double* sm_clock_mhz);
/* Random 8-byte gathers per second from a device table of 2^log2_entries
 * u64 (10..34), addresses independent of the data: the ceiling of the
 * SATOSTOP joins' gathers (measurement aid; allocates and frees the table). */
int nsat_probe_gather_peak(nsat_ctx* ctx, uint32_t log2_entries, double* gathers_per_s);

#ifdef __cplusplus
}
#endif
#endif

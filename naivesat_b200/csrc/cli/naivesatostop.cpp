// naivesatostop -- SATOSTOP (bounded halting x SAT) for a circuit with n
// inputs and n+1 outputs (drop-in for the reference's naivesatostop,
// src/satostop.rs).
//
// Same arguments (satostop.rs:62-99).  The reference's lossy hashmap of path
// segments is replaced by the next-state table and distance-carrying pointer
// doubling; -H/-U/-P/-C (hashmap tuning) are accepted and have no effect.
// Answer lines (satostop.rs:1718-1749): "Solution: Solution { start: S, end:
// E, steps: K }" or "Unsatisfiable!"; -v replays the path ("Verified: end=E
// steps=K", "INCORRECT" on a mismatch).  -S prints the simple_solve line
// "Stopped at <unknowns, decimal> <end, decimal>" (satostop.rs:1751-1782).
// The start reported is the lowest unknown assignment whose run stops
// (the order of simple_solve).
#include "cli_common.h"

using namespace cli;

int main(int argc, char** argv) {
    Args a;
    a.about = "Solve SATOSTOP with a next-state table and pointer doubling on a CUDA device";
    a.pos("CIRCUIT");
    a.pos("UNKNOWNS");
    a.flag("S", "simple", "Not real mode");
    a.option("e", "elem-inputs", "Power of two of number of elements executed at call [default: 24]");
    a.option("H", "hashmap-len-bits", "Power of two of size of hashmap [default: 24] (no effect)");
    a.option("U", "unknown-fill-bits", "(no effect)");
    a.option("P", "max-predecessors", "(no effect) [default: 0]");
    a.option("C", "iters-per-clear-predecessors", "(no effect) [default: 20]");
    a.option("t", "exec-type", "Execution type: {cpu,opencl:{dev}}");
    a.flag("n", "no-optimize-negs", "Disable optimize_negs");
    a.option("G", "opencl-group-len", "OpenCL group length (CUDA block size)");
    a.flag("v", "verify", "Verify if solution found");
    a.parse(argc, argv);
    printf("CUDA devices: %d\n", nsat_device_count());
    Loaded L;
    load_circuit(a.positional[0], &L);
    const uint32_t n = L.d.input_len;
    char* endp = nullptr;
    const unsigned long unknowns = strtoul(a.positional[1].c_str(), &endp, 10);
    if (!endp || *endp) die("invalid UNKNOWNS", 2);
    if (L.d.output_num != n + 1) die("circuit must have input_len + 1 outputs", 1);
    if (unknowns > n) die("unknowns must not exceed input_len", 1);
    const bool simple = a.has("simple");
    if (!simple) {
        if (!a.has("exec-type")) die("the following required arguments were not provided: --exec-type <EXEC_TYPE>");
        if (n < 10) die("Unsupported!", 101);
    }
    int dev = 0;
    if (a.has("exec-type")) dev = parse_exec_type(a.get("exec-type")).devices[0];
    if (n > 31) die("state longer than 31 bits is not supported with step counts", 1);
    nsat_ctx* ctx = open_ctx(dev, a);
    nsat_circuit* c = nullptr;
    check(ctx, nsat_circuit_new(ctx, &L.d, &c), "circuit");
    if (!simple) {
        printf("Unknowns: %lu\n", unknowns);
        printf("Execute in CUDA device=%d\n", dev);
    }
    const double t0 = now_s();
    nsat_table* t = nullptr;
    nsat_table_opts to{};
    to.want_steps = 1;
    check(ctx, nsat_stop_table_build(ctx, c, &to, &t), "table build");
    nsat_stop_opts so{};
    so.unknowns = (uint32_t)unknowns;
    so.mode = 1;
    nsat_stop_result r{};
    check(ctx, nsat_stop_solve(ctx, t, &so, &r), "stop solve");
    if (simple) {
        if (r.found)
            printf("Stopped at %s %s\n", decimal_padded(r.start >> (n - unknowns), unknowns).c_str(),
                   decimal_padded(r.end, n).c_str());
        else
            printf("Unsatisfiable!\n");
    } else {
        printf("Time: %.6f\n", now_s() - t0);
        if (r.found) {
            printf("Solution: Solution { start: %llu, end: %llu, steps: %llu }\n", (unsigned long long)r.start,
                   (unsigned long long)r.end, (unsigned long long)r.steps);
            if (a.has("verify")) {
                uint64_t state = r.start, steps = 0;
                const uint64_t limit = (1ull << n) + 1;
                std::vector<uint8_t> in(n);
                for (uint64_t k = 0; k < limit; k++) {
                    for (uint32_t b = 0; b < n; b++) in[b] = (uint8_t)((state >> b) & 1);
                    std::vector<uint8_t> o = eval_scalar(L.d, in);
                    uint64_t nx = 0;
                    for (uint32_t b = 0; b < n; b++) nx |= (uint64_t)o[b] << b;
                    state = nx;
                    steps++;
                    if (o[n]) break;
                }
                printf("Verified: end=%llu steps=%llu\n", (unsigned long long)state, (unsigned long long)steps);
                if (r.end != state || r.steps != steps) printf("INCORRECT\n");
            }
        } else {
            printf("Unsatisfiable!\n");
        }
    }
    nsat_table_free(t);
    nsat_circuit_free(c);
    nsat_destroy(ctx);
    return 0;
}

// naiveqsat -- decides Q0 x0 Q1 x1 ... circuit(x) == 1 for a one-output Gate
// circuit with quantifiers (drop-in for the reference's naiveqsat,
// src/qsat.rs).
//
// Same arguments (qsat.rs:74-96); the answer line follows FinalResult's
// Display (qsat.rs:156-170): "Result: (Satisfiable: <bits>)",
// "Result: (Unsatisfiable)", "Result: (Unsatisfiable: <bits>)" or
// "Result: (Satisfiable)"; <bits> is the first quantifier block, input k at
// bit k, printed most significant first.  A file that does not parse as a
// quantified circuit is read as a plain circuit with every input existential
// (qsat.rs:6277-6285).
#include "cli_common.h"

using namespace cli;

int main(int argc, char** argv) {
    Args a;
    a.about = "Solve QSAT for a one-output Gate circuit by exhaustive search on CUDA devices";
    a.pos("CIRCUIT");
    a.option("e", "elem-inputs", "Power of two of number of elements executed at call [default: 24]");
    a.option("t", "exec-type", "Execution type: {cpu|opencl:{dev},cpu_and_openclXX}");
    a.flag("n", "no-optimize-negs", "Disable optimize_negs");
    a.option("G", "opencl-group-len", "OpenCL group length (CUDA block size)");
    a.parse(argc, argv);
    if (!a.has("exec-type")) die("the following required arguments were not provided: --exec-type <EXEC_TYPE>");
    printf("CUDA devices: %d\n", nsat_device_count());
    Loaded L;
    load_circuit(a.positional[0], &L);
    const uint32_t n = L.d.input_len;
    std::vector<uint8_t> quants(n, 0);
    if (L.quants) quants.assign(L.quants, L.quants + n);
    if (L.d.output_num != 1) die("circuit must have exactly one output", 1);
    uint32_t chunk_bits = 0;
    if (n >= 14) {
        uint32_t e = (uint32_t)a.num("elem-inputs", 24);
        if (e >= n) e = n - 1;
        if (!(e > 12 && e <= 64)) die("elem_inputs must be in 13..64", 1);
        if (!(n - e > 0 && n - e <= 64)) die("input_len - elem_inputs must be in 1..64", 1);
        printf("Elem inputs: %u\n", e);
        if (a.has("elem-inputs")) chunk_bits = e;
    }
    ExecType et = parse_exec_type(a.get("exec-type"));
    printf("Execute in CUDA device=%d\n", et.devices[0]);
    nsat_ctx* ctx = open_ctx(et.devices[0], a);
    nsat_circuit* c = nullptr;
    check(ctx, nsat_circuit_new(ctx, &L.d, &c), "circuit");
    nsat_qsat_opts o{};
    o.chunk_bits = chunk_bits;
    nsat_qsat_result r{};
    printf("Start execution\n");
    fflush(stdout);
    const double t0 = now_s();
    check(ctx, nsat_qsat_solve(ctx, c, quants.data(), &o, &r), "qsat solve");
    printf("Time: %.6f\n", now_s() - t0);
    const u128 sol = ((u128)r.solution_hi << 64) | r.solution_lo;
    std::string s;
    if (r.reversed) s = r.has_solution ? "(Unsatisfiable: " + binary(sol, r.solution_bits) + ")" : "(Satisfiable)";
    else s = r.has_solution ? "(Satisfiable: " + binary(sol, r.solution_bits) + ")" : "(Unsatisfiable)";
    printf("Result: %s\n", s.c_str());
    nsat_circuit_free(c);
    nsat_destroy(ctx);
    return 0;
}

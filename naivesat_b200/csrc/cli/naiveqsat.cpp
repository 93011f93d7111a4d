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
// (qsat.rs:6277-6285).  The combined exec types split the outermost
// log2(devices) quantifiers over all visible devices, one host thread and
// context per device, and join the sub-answers with a forall/exists reducer.
#include <thread>

#include "../qreducer.h"
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
    // shard over a power-of-two number of devices on the outermost inputs
    uint32_t sbits = 0;
    while ((1u << (sbits + 1)) <= et.devices.size() && sbits + 1 + 14 <= n) sbits++;
    const size_t D = (size_t)1 << sbits;
    if (D == 1) printf("Execute in CUDA device=%d\n", et.devices[0]);
    else printf("Execute in %zu CUDA devices (outermost %u inputs split)\n", D, sbits);
    std::vector<nsat_qsat_result> subs(D);
    std::vector<int> rcs(D, 0);
    std::vector<std::string> errs(D);
    printf("Start execution\n");
    fflush(stdout);
    const double t0 = now_s();
    std::vector<std::thread> th;
    for (size_t i = 0; i < D; i++) {
        th.emplace_back([&, i]() {
            nsat_ctx* ctx = open_ctx(et.devices[i], a);
            nsat_circuit* c = nullptr;
            int rc = nsat_circuit_new(ctx, &L.d, &c);
            if (rc == NSAT_OK) rc = maybe_autotune(ctx, c, 1, quants.data());
            if (rc == NSAT_OK) {
                nsat_qsat_opts o{};
                o.chunk_bits = chunk_bits;
                o.prefix_bits = sbits;
                o.prefix = i;
                rc = nsat_qsat_solve(ctx, c, quants.data(), &o, &subs[i]);
            }
            rcs[i] = rc;
            if (rc) errs[i] = nsat_last_error(ctx);
            nsat_circuit_free(c);
            nsat_destroy(ctx);
        });
    }
    for (auto& t : th) t.join();
    for (size_t i = 0; i < D; i++)
        if (rcs[i]) die(std::string("qsat solve: ") + nsat_strerror(rcs[i]) + " " + errs[i], 1);
    nsat_qsat_result r = subs[0];
    if (D > 1) {
        // forall/exists over the split inputs, sub-answers in prefix order
        uint32_t f = 0;
        while (f < n && quants[f] == quants[0]) f++;
        nsat::QuantReducer qr(std::vector<uint8_t>(quants.begin(), quants.begin() + sbits));
        nsat::FinalResult fr;
        for (size_t i = 0; i < D; i++) {
            const bool value = (subs[i].has_solution != 0) != (subs[i].reversed != 0);
            qr.push(value);
            if (!qr.final_result(&fr)) continue;
            r.reversed = quants[0];
            r.solution_bits = f;
            r.has_solution = fr.has_solution;
            u128 sol = fr.solution;
            if (fr.has_solution && f > sbits) sol |= ((u128)subs[i].solution_lo) << sbits;
            r.solution_lo = (uint64_t)sol;
            r.solution_hi = (uint64_t)(sol >> 64);
            break;
        }
    }
    printf("Time: %.6f\n", now_s() - t0);
    const u128 sol = ((u128)r.solution_hi << 64) | r.solution_lo;
    std::string s;
    if (r.reversed) s = r.has_solution ? "(Unsatisfiable: " + binary(sol, r.solution_bits) + ")" : "(Satisfiable)";
    else s = r.has_solution ? "(Satisfiable: " + binary(sol, r.solution_bits) + ")" : "(Unsatisfiable)";
    printf("Result: %s\n", s.c_str());
    return 0;
}

// naivesat -- finds an input vector for which a one-output Gate circuit
// returns 1 (drop-in for the reference's naivesat, src/main.rs).
//
// Same arguments (main.rs:52-74) and answer lines (main.rs:373-381):
//   "Found Input: <n binary digits, input n-1 first>", "Unsatisfiable!",
//   "INCORRECT!! <bits>" if the witness fails the scalar re-check.
// The witness is the lowest satisfying index (input b = bit b).  Every exec
// type runs on CUDA devices; the combined types split the index space over
// all visible devices, one host thread and context per device.
#include <thread>

#include "cli_common.h"

using namespace cli;

int main(int argc, char** argv) {
    Args a;
    a.about = "Solve SAT for a one-output Gate circuit by exhaustive search on CUDA devices";
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
    if (L.d.output_num != 1) die("circuit must have exactly one output", 1);
    uint32_t chunk_bits = 0;   // auto: 2^34 assignments per launch
    if (n >= 14) {
        uint32_t e = (uint32_t)a.num("elem-inputs", 24);
        if (e >= n) e = n - 1;
        if (!(e > 12 && e <= 64)) die("elem_inputs must be in 13..64", 1);
        if (!(n - e > 0 && n - e <= 64)) die("input_len - elem_inputs must be in 1..64", 1);
        printf("Elem inputs: %u\n", e);
        if (a.has("elem-inputs")) chunk_bits = e;
    }
    ExecType et = parse_exec_type(a.get("exec-type"));
    printf("Execute in %s\n", et.label.c_str());
    // every device claims launches from one shared queue over the whole
    // range and stops once any of them holds a witness below its next claim
    // (the reference's ParSeq mapper, main.rs:205-264)
    const size_t D = et.devices.size();
    nsat_sat_share share{};
    std::vector<nsat_sat_result> res(D);
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
            if (rc == NSAT_OK) rc = maybe_autotune(ctx, c, 0, nullptr);
            if (rc == NSAT_OK) {
                nsat_sat_opts o{};
                o.find_all = 0;
                o.chunk_bits = chunk_bits;
                o.share = D > 1 ? &share : nullptr;
                rc = nsat_sat_solve(ctx, c, &o, &res[i]);
            }
            rcs[i] = rc;
            if (rc) errs[i] = nsat_last_error(ctx);
            nsat_circuit_free(c);
            nsat_destroy(ctx);
        });
    }
    for (auto& t : th) t.join();
    for (size_t i = 0; i < D; i++)
        if (rcs[i]) die(std::string("sat solve: ") + nsat_strerror(rcs[i]) + " " + errs[i], 1);
    printf("Time: %.6f\n", now_s() - t0);
    bool found = false;
    u128 w = 0;
    for (size_t i = 0; i < D; i++) {
        if (!res[i].satisfiable) continue;
        const u128 wi = ((u128)res[i].witness_hi << 64) | res[i].witness_lo;
        if (!found || wi < w) w = wi;
        found = true;
    }
    if (found) {
        std::vector<uint8_t> in(n);
        for (uint32_t b = 0; b < n; b++) in[b] = (uint8_t)((w >> b) & 1);
        if (!eval_scalar(L.d, in)[0]) printf("INCORRECT!! %s\n", binary(w, n).c_str());
        else printf("Found Input: %s\n", binary(w, n).c_str());
    } else {
        printf("Unsatisfiable!\n");
    }
    return 0;
}

// greedysatostop -- SATOSTOP by a full next-state table and pointer-doubling
// joins (drop-in for the reference's greedysatostop, src/greedysatostop.rs).
//
// Same arguments (greedysatostop.rs:28-49).  The circuit has n inputs and
// n+1 outputs (outputs 0..n-1 = next state, output n = STOP); the unknowns
// are the top `unknowns` state bits.  Answer lines (greedysatostop.rs:
// 1110-1137): "Solution: Solution { start: S, end: E }" or "Unsatisfiable!";
// with -v the path is replayed: "Verified: end=E" and "INCORRECT" on a
// mismatch.  The table lives in device memory (two ping-pong buffers); the
// start reported is the lowest one among those resolved in the first
// doubling round that resolves any.  With -p P the table is a packed image
// outside device memory (pinned host memory, or with -x PREFIX the temp file
// PREFIXgreedy_temp_<ns>) joined partition by partition in the reference's
// order (greedysatostop.rs:692-837), so the answer is the reference's for
// that P.
#include "cli_common.h"

using namespace cli;

int main(int argc, char** argv) {
    Args a;
    a.about = "Solve SATOSTOP with a next-state table and pointer doubling on a CUDA device";
    a.pos("CIRCUIT");
    a.pos("UNKNOWNS");
    a.option("C", "opencl", "CUDA device to execute circuits on [default: 0]");
    a.flag("n", "no-optimize-negs", "Disable optimize_negs");
    a.option("p", "partitions", "Partitions that can be used if too small memory");
    a.option("x", "file-image-prefix", "Prefix of the table spill file");
    a.flag("v", "verify", "Verify if solution found");
    a.parse(argc, argv);
    printf("CUDA devices: %d\n", nsat_device_count());
    Loaded L;
    load_circuit(a.positional[0], &L);
    const uint32_t n = L.d.input_len;
    char* end = nullptr;
    const unsigned long unknowns = strtoul(a.positional[1].c_str(), &end, 10);
    if (!end || *end) die("invalid UNKNOWNS", 2);
    if (L.d.output_num != n + 1) die("circuit must have input_len + 1 outputs", 1);
    if (unknowns > n) die("unknowns must not exceed input_len", 1);
    if (n >= 64) die("input_len must be below 64", 1);
    uint64_t parts = 0;
    if (a.has("partitions")) {
        parts = a.num("partitions", 0);
        if (a.has("opencl")) die("partitions run without -C (the reference asserts this)", 101);
        if (parts < 2) die("Too small number of partitions", 101);
        if (parts & (parts - 1)) die("Number of partitions must be power of 2", 101);
        uint32_t pb = 0;
        while ((1ull << pb) < parts) pb++;
        printf("Load partition bits: %u\n", std::min<uint32_t>(pb + 2, n - 10));
    }
    const int dev = (int)a.num("opencl", 0);
    nsat_ctx* ctx = open_ctx(dev, a);
    nsat_circuit* c = nullptr;
    check(ctx, nsat_circuit_new(ctx, &L.d, &c), "circuit");
    const double t0 = now_s();
    printf("Calculate first nexts\n");
    nsat_table* t = nullptr;
    nsat_stop_result r{};
    if (parts) {
        nsat_greedy_opts go{};
        go.unknowns = (uint32_t)unknowns;
        go.partitions = (uint32_t)parts;
        const std::string prefix = a.has("file-image-prefix") ? a.get("file-image-prefix") : std::string();
        go.file_prefix = a.has("file-image-prefix") ? prefix.c_str() : nullptr;
        nsat_greedy_result gr{};
        check(ctx, nsat_greedy_solve(ctx, c, &go, &gr), "partitioned solve");
        printf("Joined %llu partition pairs\n", (unsigned long long)gr.joins);
        r.found = gr.found;
        r.start = gr.start;
        r.end = gr.end;
    } else {
        nsat_table_opts to{};
        check(ctx, nsat_stop_table_build(ctx, c, &to, &t), "table build");
        nsat_stop_opts so{};
        so.unknowns = (uint32_t)unknowns;
        so.mode = 0;
        check(ctx, nsat_stop_solve(ctx, t, &so, &r), "stop solve");
        printf("Joining nexts: %u stages\n", r.rounds);
    }
    printf("Time: %.6f\n", now_s() - t0);
    if (r.found) {
        printf("Solution: Solution { start: %llu, end: %llu }\n", (unsigned long long)r.start,
               (unsigned long long)r.end);
        if (a.has("verify")) {
            uint64_t state = r.start;
            const uint64_t limit = n < 63 ? (1ull << n) + 1 : ~0ull;
            std::vector<uint8_t> in(n);
            for (uint64_t k = 0; k < limit; k++) {
                for (uint32_t b = 0; b < n; b++) in[b] = (uint8_t)((state >> b) & 1);
                std::vector<uint8_t> o = eval_scalar(L.d, in);
                uint64_t nx = 0;
                for (uint32_t b = 0; b < n; b++) nx |= (uint64_t)o[b] << b;
                state = nx;
                if (o[n]) break;
            }
            printf("Verified: end=%llu\n", (unsigned long long)state);
            if (r.end != state) printf("INCORRECT\n");
        }
    } else {
        printf("Unsatisfiable!\n");
    }
    if (t) nsat_table_free(t);
    nsat_circuit_free(c);
    nsat_destroy(ctx);
    return 0;
}

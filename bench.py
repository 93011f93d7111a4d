#!/usr/bin/env python3
"""Benchmark of the naivesat hot path on B200.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                  [--workload c1|c0|c1_twin|c2a|c2b|c2c|c3a|c3b|c3m|c3s|c3p|c3p_spill|c4]

Default workload (c1): exhaustive bit-sliced SAT of the 36-input / 3018-gate
planted random-DAG circuit (seed 1), exact solution count plus lowest witness
over all 2^36 assignments.  One step = one full enumeration, the index space
split evenly across the N ranks (one GPU each); a tiny all-reduce combines
counts and times.  `value` is device time (CUDA events around every kernel
launch on the launching stream), `e2e` the same work through the C ABI call
from host buffers (circuit upload, launches, result readback); both are the
max over ranks.  `--impl reference` times the oracle port of the reference's
gatenative CPU path on this host's cores instead (rank 0 only).

The other workloads print the same line shape for the QSAT (c2*) and
SATOSTOP (c3*) paths; their steps are replicas on every rank.  c4 is the
serving trace (10,000 requests): `value` is solves/s with every request
queued at t=0, `latency` the p50/p99 under Poisson arrivals, `plain` the
one-launch-per-instance form on the same trace.
"""
import argparse
import json
import math
import os
import shutil
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)


def dist_setup():
    import torch
    import torch.distributed as dist
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        backend = "nccl" if torch.cuda.is_available() else "gloo"
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=timedelta(seconds=600))
    return world, rank, local


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None

    def start(self):
        if not shutil.which("nvidia-smi"):
            return
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        self.f = open(self.path, "w")
        self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.device), "--query-gpu=" + self.Q,
                                      "--format=csv,noheader,nounits", "-lms", "200"],
                                     stdout=self.f, stderr=subprocess.DEVNULL)
        # a region shorter than the sampling period still gets a sample on
        # each side: wait for the first one before the region starts
        self.lines_at_start = self._wait_lines(1, 5.0)

    def _wait_lines(self, n, limit_s):
        t0 = time.time()
        while time.time() - t0 < limit_s:
            self.f.flush()
            try:
                with open(self.path) as f:
                    k = sum(1 for _ in f)
            except OSError:
                k = 0
            if k >= n:
                return k
            time.sleep(0.02)
        return 0

    def stop(self):
        if not self.proc:
            return None
        self._wait_lines(self.lines_at_start + 1, 1.0)     # and one after it ends
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) < 9:
                continue
            try:
                sm.append(float(p[1]))
                mx = max(mx, float(p[2]))
            except ValueError:
                continue
            for nm, v in zip(names, p[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        os.unlink(self.path)
        if not sm:
            return None
        loaded = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(loaded), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def cpu_model():
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def measured_hbm_gbs():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# --------------------------------------------------------------------------
# workloads

class SatWorkload:
    """Exhaustive SAT: count + lowest witness over 2^min(n, log2) assignments."""
    metric = "gate-evals/s"
    kind = "sat"

    def __init__(self, name, log2):
        from naivesat_b200 import workloads as W
        self.name = name
        self.circ = W.config(name)
        self.total = 1 << min(self.circ.n, log2)

    def describe(self):
        c = self.circ
        return {"workload": "naivesat %s: %d-input %d-gate random DAG (%s), exhaustive SAT over "
                            "2^%d assignments, exact count + lowest witness"
                            % (self.name, c.n, c.num_gates, c.name, int(math.log2(self.total))),
                "inputs": c.n, "gates": c.num_gates, "assignments_per_step": self.total}

    def setup(self, ctx, world, rank):
        per = self.total // world
        self.begin, self.end = rank * per, (rank + 1) * per
        self.ctx = ctx
        self.h = ctx.circuit(self.circ)
        self.live, self.lop3 = self.h.stats()

    def step(self, fresh=False):
        h = self.ctx.circuit(self.circ) if fresh else self.h
        r = h.sat(find_all=True, begin=self.begin, end=self.end)
        return {"device_ms": r["device_ms"], "launches": r["launches"],
                "sig": (r["count"], r["witness"]), "count": r["count"], "witness": r["witness"]}

    def work(self):           # gate-evals per step (all ranks)
        return self.total * self.circ.num_gates

    def roofline(self, world, dev_ms_per_step, peak_lop3, probe_mhz):
        words = (self.total // world) // 32
        rate = words * self.lop3 / (dev_ms_per_step * 1e-3)
        return {"bound": "alu", "achieved": rate, "peak": peak_lop3, "unit": "lop3/s",
                "frac": rate / peak_lop3, "traffic": 212736,
                "traffic_note": "dram bytes per launch from ncu on a 2^32 launch (instruction and "
                                "parameter fetch only; the kernel reads no data)",
                "peak_source": "measured lop3.b32 chain microbenchmark on this GPU (%.0f MHz)" % probe_mhz,
                "lop3_per_word": self.lop3, "live_gates": self.live}

    def cpu(self, threads, target_s=12.0):
        """The generated-code CPU path (oracle/cpu_codegen.py) on a bounded
        sample, plus the oracle's interpreter on a smaller one for the factor
        between the two."""
        g = cpu_codegen_sat(self.circ)
        per, span, dt = time_codegen_sample(g, threads, target_s / 3)
        rate = per * self.circ.num_gates / dt
        irate, isample = interpreter_rate(self.circ, threads, 3.0)
        g.close()
        return rate, ("generated C per circuit, %d-bit vectors, gcc -O3 -march=native, OpenMP over args of "
                      "2^%d assignments; %s in %.1f s" % (g.vector_bits, g.e, span, dt)), \
            {"method": "codegen", "interpreter_value": irate, "interpreter_sample": isample,
             "codegen_over_interpreter": rate / irate}


class QsatWorkload:
    """QSAT decision + first-block witness (early exit as the tree allows)."""
    metric = "gate-evals/s"
    kind = "qsat"

    def __init__(self, name):
        from naivesat_b200 import workloads as W
        self.name = name
        self.circ = W.config(name)

    def describe(self):
        c = self.circ
        return {"workload": "naiveqsat %s: %d inputs, %d gates, quantifiers %s" % (self.name, c.n, c.num_gates,
                                                                               c.quants),
                "inputs": c.n, "gates": c.num_gates}

    def setup(self, ctx, world, rank):
        self.ctx = ctx
        self.h = ctx.circuit(self.circ)
        self.live, self.lop3 = self.h.stats()
        self.scanned = None

    def step(self, fresh=False):
        h = self.ctx.circuit(self.circ) if fresh else self.h
        r = h.qsat(self.circ.quants)
        self.scanned = r["scanned"]
        return {"device_ms": r["device_ms"], "launches": r["launches"],
                "sig": (r["reversed"], r["solution_bits"], r["solution"]), "result": r}

    def work(self):
        return self.scanned * self.circ.num_gates

    def roofline(self, world, dev_ms_per_step, peak_lop3, probe_mhz):
        rate = (self.scanned // 32) * self.lop3 / (dev_ms_per_step * 1e-3)
        return {"bound": "alu", "achieved": rate, "peak": peak_lop3, "unit": "lop3/s",
                "frac": rate / peak_lop3, "traffic": None,
                "peak_source": "measured lop3.b32 chain microbenchmark on this GPU (%.0f MHz)" % probe_mhz,
                "lop3_per_word": self.lop3, "live_gates": self.live}

    def cpu(self, threads, target_s=12.0):
        """The reference's CPU QSAT path restated as generated C (oracle/
        cpu_codegen.py: per-circuit vector code in v-order, calls reduced to
        their first-block units, the first block's QuantReducer), full solves
        repeated for about target_s / 3; beside it the oracle's interpreter
        (one QuantReducer push per item) for the factor between the two.
        The two FinalResults must agree."""
        from oracle import cpu_codegen as CG, oracle as O
        oc = O.Circuit(self.circ.n, self.circ.gates, self.circ.outputs)
        work = (1 << self.circ.n) * self.circ.num_gates
        t0 = time.perf_counter()
        ref = O.qsat(oc, self.circ.quants, mode=1, threads=threads)
        dti = time.perf_counter() - t0
        irate = work / dti
        try:
            g = CG.CodegenQsat(self.circ, self.circ.quants)
        except ValueError:      # units smaller than a vector word: the interpreter only
            return irate, "full oracle solve (%.1f s)" % dti
        reps, dt = 0, 0.0
        while reps < 1 or (dt < target_s / 3 and reps < 200):
            t0 = time.perf_counter()
            got = g.solve(threads)
            dt += time.perf_counter() - t0
            reps += 1
        g.close()
        assert got == ref, (got, ref)
        rate = reps * work / dt
        return rate, ("generated C per circuit, %d-bit vectors, gcc -O3 -march=native, OpenMP over args of 2^%d "
                      "items, first-block QuantReducer over the calls' units; %d full solve(s) in %.2f s"
                      % (g.vector_bits, g.e, reps, dt)), \
            {"method": "codegen", "interpreter_value": irate,
             "interpreter_sample": "full oracle solve (%.1f s)" % dti, "codegen_over_interpreter": rate / irate}


def gather_roofline(ctx, log2_table, gathers, stream_bytes, ms, hbm_gbs):
    """A join is one random gather per entry plus streaming reads/writes:
    its ceiling is gathers / (measured random-gather rate over a table of the
    same size) + stream_bytes / (measured copy bandwidth)."""
    g = ctx.gather_peak(min(34, max(10, log2_table)))
    t = gathers / g + stream_bytes / (hbm_gbs * 1e9)
    return {"gathers_per_s_peak": g, "table_log2": log2_table, "ceiling_ms": t * 1e3, "achieved_ms": ms,
            "frac": t * 1e3 / ms,
            "note": "gather peak: nsat_probe_gather_peak, independent random 8-byte loads over a table of "
                    "2^table_log2 u64; streaming at the measured copy bandwidth"}


class StopWorkload:
    """SATOSTOP: table build + synchronous doubling, both on the device."""
    metric = "join GB/s"
    kind = "stop"

    def __init__(self, name, unknowns, mode, steps_counts):
        from naivesat_b200 import workloads as W
        self.name = name
        if name == "c3s":
            self.circ = W.lfsr_stop(4, 32, 300)
        elif name == "c3m":
            self.circ = W.lfsr_stop(4, 28, 300)
        else:
            self.circ = W.config(name)
        self.u, self.mode, self.want_steps = unknowns, mode, steps_counts

    def describe(self):
        c = self.circ
        return {"workload": "SATOSTOP %s: %d-bit state, %d unknowns, %d gates, table + pointer doubling "
                            "(mode %d)" % (self.name, c.n, self.u, c.num_gates, self.mode),
                "state_bits": c.n, "unknowns": self.u, "gates": c.num_gates,
                "entry_bytes": 8 if (self.want_steps or c.n > 31) else 4}

    def setup(self, ctx, world, rank):
        self.ctx = ctx
        self.h = ctx.circuit(self.circ)
        self.rounds = None
        self.eb = 8 if (self.want_steps or self.circ.n > 31) else 4

    def step(self, fresh=False):
        h = self.ctx.circuit(self.circ) if fresh else self.h
        t = h.stop_table(want_steps=self.want_steps)
        r = t.solve(self.u, mode=self.mode)
        del t
        self.rounds = r["rounds"]
        self.join_ms = r["join_ms"]
        self.build_ms = r["build_ms"]
        return {"device_ms": r["build_ms"] + r["join_ms"], "launches": 1 + self.circ.n,
                "sig": (r["found"], r.get("start"), r.get("end"), r.get("steps"), r["rounds"]), "result": r}

    def join_bytes(self):
        return self.rounds * (1 << self.circ.n) * 3 * self.eb

    def work(self):
        return self.join_bytes() / 1e9

    def roofline(self, world, dev_ms_per_step, peak_lop3, probe_mhz):
        peak, src = measured_hbm_gbs()
        ach = self.join_bytes() / (self.join_ms * 1e-3) / 1e9
        out = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak,
               "traffic": None, "peak_source": "%s hbm_gbs (MEASURED_PEAKS.json)" % src,
               "kernel": "join_round", "algorithmic_bytes_per_entry_round": 3 * self.eb,
               "rounds": self.rounds, "join_ms": self.join_ms, "build_ms": self.build_ms}
        # probe table of the same bytes as this table (u64 probe entries)
        out["gather_roofline"] = gather_roofline(self.ctx, self.circ.n - (1 if self.eb == 4 else 0),
                                                 (1 << self.circ.n) * self.rounds,
                                                 (1 << self.circ.n) * self.rounds * 2 * self.eb, self.join_ms, peak)
        return out

    def cpu(self, threads, target_s=12.0):
        from oracle import oracle as O
        if self.circ.n > 26:
            return None, "state too large for the host oracle"
        oc = O.Circuit(self.circ.n, self.circ.gates, self.circ.outputs)
        t0 = time.perf_counter()
        tb = O.stop_table(oc, threads)
        r = O.stop_solve(self.circ.n, self.u, tb, mode=self.mode, threads=threads)
        dt = time.perf_counter() - t0
        rounds = r["rounds"] if r else self.circ.n
        bytes_ = rounds * (1 << self.circ.n) * 3 * 8
        return bytes_ / dt / 1e9, "full oracle table + doubling (%.1f s, u64 arrays)" % dt


class StopPartWorkload:
    """Partitioned greedysatostop (-p): packed (n+1)-bit image, partition
    joins in the reference's order; the image in device memory (c3p) or
    spilled to pinned host memory (c3p_spill)."""
    metric = "join GB/s"
    kind = "stop"

    def __init__(self, name):
        from naivesat_b200 import workloads as W
        self.name = name
        self.n, self.u, self.P = 28, 20, 4
        self.circ = W.lfsr_stop(4, self.n, 300)
        self.spill = name.endswith("spill")

    def describe(self):
        c = self.circ
        return {"workload": "greedysatostop -p %d %s: %d-bit LFSR state, %d unknowns, %d gates, packed %d-bit "
                            "image %s" % (self.P, self.name, c.n, self.u, c.num_gates, c.n + 1,
                                          "in pinned host memory (PCIe per partition)" if self.spill else
                                          "in device memory"),
                "state_bits": c.n, "unknowns": self.u, "partitions": self.P, "gates": c.num_gates}

    def setup(self, ctx, world, rank):
        self.ctx = ctx
        self.h = ctx.circuit(self.circ)

    def step(self, fresh=False):
        h = self.ctx.circuit(self.circ) if fresh else self.h
        r = h.greedy_partitioned(self.u, self.P, device_bytes=1 if self.spill else 0)
        self.last = r
        ms = r["build_ms"] + r["join_ms"] if not self.spill else r["wall_ms"]
        return {"device_ms": ms, "launches": int(r["joins"]) * 2 + (1 << r["load_bits"]) * 2,
                "sig": (r["found"], r["start"], r["end"], r["stage"], r["partition"]), "result": r}

    def join_bytes(self):
        # per join launch: every entry of dest is read (8 B); the entries whose
        # next state lies in the joined partition, 1/P of them for uniformly
        # spread next states, gather one entry and write dest (8 + 8 B)
        return self.last["joins"] * (1 << (self.n - 2)) * (8 + 16 / self.P)

    def work(self):
        return self.join_bytes() / 1e9

    def roofline(self, world, dev_ms_per_step, peak_lop3, probe_mhz):
        peak, src = measured_hbm_gbs()
        r = self.last
        ach = self.join_bytes() / (r["join_ms"] * 1e-3) / 1e9
        out = {"bound": "hbm", "achieved": ach, "peak": peak, "unit": "GB/s", "frac": ach / peak, "traffic": None,
               "peak_source": "%s hbm_gbs (MEASURED_PEAKS.json)" % src, "kernel": "join_packed_kernel",
               "algorithmic_bytes_per_entry_join": 8 + 16 / self.P,
               "joins": r["joins"], "join_ms": r["join_ms"], "build_ms": r["build_ms"], "wall_ms": r["wall_ms"],
               "storage": ["device", "pinned host", "file"][r["storage"]]}
        if self.spill:
            out["pcie_gbs"] = (r["h2d_bytes"] + r["d2h_bytes"]) / (r["wall_ms"] * 1e-3) / 1e9
        L = 1 << (self.n - 2)
        # per join: L/P gathers from the packed partition (~L*(n+1)/8 bytes, i.e. 2^(n-3) u64 of table),
        # 8 B read per entry, 8 B written per gathered entry
        out["gather_roofline"] = gather_roofline(self.ctx, self.n - 3, r["joins"] * L / self.P,
                                                 r["joins"] * (8 * L + 8 * L / self.P), r["join_ms"], peak)
        return out

    def cpu(self, threads, target_s=12.0):
        return None, "the oracle's partitioned schedule runs on packed entries one at a time; n=28 is out of reach"


def cpu_codegen_sat(circ):
    from oracle import cpu_codegen as CG
    return CG.CodegenSat(circ, 24)


def time_codegen_sample(g, threads, min_s, start_arg=0):
    """Times whole calls of the generated SAT evaluator: args from start_arg,
    doubling their number until one timed pass takes min_s (the whole index
    space at most, repeated when that is faster).  Returns (assignments,
    description, seconds)."""
    nargs = 1 << (g.circ.n - g.e)
    k = 1
    while True:
        a0 = start_arg % nargs
        a1 = min(nargs, a0 + k)
        reps = 0
        t0 = time.perf_counter()
        while True:
            g.sat_args(a0, a1, threads)
            reps += 1
            dt = time.perf_counter() - t0
            if a1 - a0 < k and dt < min_s:
                continue          # the whole space is smaller than the sample: repeat it
            break
        if dt >= min_s or (a1 - a0) < k:
            span = "%d pass(es) over args [%d, %d)" % (reps, a0, a1)
            return reps * ((a1 - a0) << g.e), span, dt
        k *= 2


def interpreter_rate(circ, threads, min_s):
    """The oracle's slot interpreter (the checker) over the first 2^k
    assignments, k growing until a pass takes min_s / 3."""
    from oracle import oracle as O
    oc = O.Circuit(circ.n, circ.gates, circ.outputs)
    bits = min(20, circ.n)
    while True:
        t0 = time.perf_counter()
        O.sat_range(oc, 0, 1 << bits, threads)
        dt = time.perf_counter() - t0
        if dt > min_s / 3 or bits >= circ.n:
            break
        bits += 1
    return (1 << bits) * circ.num_gates / dt, "first 2^%d assignments (%.1f s)" % (bits, dt)


def make_workload(name, log2):
    if name in ("c3p", "c3p_spill"):
        return StopPartWorkload(name)
    if name in ("c0", "c1", "c1_twin"):
        return SatWorkload(name, log2)
    if name in ("c2a", "c2b", "c2c"):
        return QsatWorkload(name)
    if name in ("c3a", "c3b"):
        return StopWorkload(name, 16, 0, False)
    if name in ("c3s", "c3m"):
        return StopWorkload(name, 20, 0, False)
    raise SystemExit("unknown workload " + name)


# --------------------------------------------------------------------------

def run_reference(args, world, rank):
    """Reference arm: the oracle port of the reference's CPU path, rank 0 only."""
    if rank != 0:
        return
    wl = make_workload(args.workload, args.log2)
    threads = os.cpu_count() or 1
    if wl.kind != "sat":
        outs = [wl.cpu(threads) for _ in range(max(1, args.steps))]
        rate = statistics.median(o[0] for o in outs)
        sample = outs[-1][1] + " per step"
        span = None
    else:
        # the reference's CPU path restated as generated C per circuit
        # (oracle/cpu_codegen.py); each step a bounded sample of args of
        # 2^e assignments, moving through the index space
        circ = wl.circ
        g = cpu_codegen_sat(circ)
        nargs = 1 << (circ.n - g.e)
        t0 = time.perf_counter()
        g.sat_args(0, 1, threads)
        one = max(time.perf_counter() - t0, 1e-4)
        k = max(1, min(nargs, int(4.0 / one)))     # about 4 s of work per step
        span = k << g.e
        times = []
        for s in range(args.warmup + args.steps):
            a0 = (s * k) % nargs
            a1 = min(nargs, a0 + k)
            t0 = time.perf_counter()
            g.sat_args(a0, a1, threads)
            if a1 - a0 < k:
                g.sat_args(0, k - (a1 - a0), threads)
            if s >= args.warmup:
                times.append(time.perf_counter() - t0)
        rate = span * circ.num_gates * args.steps / sum(times)
        sample = ("%d args of 2^%d assignments per step (2^%.1f of 2^%d), generated C per circuit with %d-bit "
                  "vectors, gcc -O3 -march=native, OpenMP over args" % (k, g.e, math.log2(span), circ.n,
                                                                        g.vector_bits))
        g.close()
    line = {"impl": "reference", "metric": wl.metric, "value": rate, "unit": wl.metric, "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": (1e3 * span * wl.circ.num_gates / rate) if span else None,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "u64 bit-sliced (vector words)", "data": "synthetic",
            "config": dict(wl.describe(), cpu=cpu_model()),
            "cpu_baseline": {"value": rate, "unit": wl.metric, "cores": threads, "kind": "port",
                             "method": "codegen" if span else "oracle",
                             "sample": sample + "; the reference's Rust/gatenative code cannot be built "
                                                "here, so its restatement in oracle/ runs it"},
            "e2e": {"value": rate, "unit": wl.metric, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_ours(args, world, rank, local):
    import torch
    from naivesat_b200 import api

    wl = make_workload(args.workload, args.log2)
    ctx = api.Context(local)
    wl.setup(ctx, world, rank)
    torch.cuda.set_device(local)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.int32, device="cuda")

    def reduce(vals, op):
        if world == 1:
            return vals
        import torch.distributed as dist
        t = torch.tensor(vals, dtype=torch.float64, device="cuda")
        dist.all_reduce(t, op=dist.ReduceOp.MAX if op == "max" else dist.ReduceOp.SUM)
        return t.tolist()

    def barrier():
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    peak_lop3, probe_mhz = ctx.lop3_peak()
    t_warm = time.perf_counter()
    ref = None
    for _ in range(args.warmup):
        ref = wl.step()
    t_warm = time.perf_counter() - t_warm

    clocks = ClockSampler(local)
    barrier()
    clocks.start()
    dev_ms, launches = [], 0
    for s in range(args.steps):
        flush.fill_(s)                    # L2 flush between steps, outside the events
        torch.cuda.synchronize()
        r = wl.step()
        dev_ms.append(r["device_ms"])
        launches += r["launches"]
        assert ref is None or r["sig"] == ref["sig"], (r["sig"], ref["sig"])
    barrier()
    clk = clocks.stop()

    barrier()
    e2e_ms = []
    for s in range(args.steps):
        t0 = time.perf_counter()
        r = wl.step(fresh=True)
        e2e_ms.append(1e3 * (time.perf_counter() - t0))
    barrier()

    tot_dev, tot_e2e = reduce([sum(dev_ms), sum(e2e_ms)], "max")
    extra = {}
    if wl.kind == "sat":
        extra["count"] = int(reduce([float(r["count"])], "sum")[0])
        extra["witness"] = r["witness"]
    if rank != 0:
        return
    steps = args.steps
    ms_step = tot_dev / steps
    value = wl.work() * steps / (tot_dev * 1e-3)
    e2e = wl.work() * steps / (tot_e2e * 1e-3)
    cold = cold_probe(args, local) if (world == 1 and not args.no_e2e_cold) else None
    if cold is not None:
        cold["value"] = wl.work() / (cold["solve_ms"] * 1e-3)
        cold["unit"] = wl.metric
    lps = launches / steps
    cpu = None
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        out = wl.cpu(threads)
        v, sample = out[0], out[1]
        if v is not None:
            cpu = {"value": v, "unit": wl.metric, "cores": threads, "kind": "port",
                   "sample": sample + ", " + cpu_model()}
            if len(out) > 2:
                cpu.update(out[2])
    cfg = wl.describe()
    cfg.update(extra)
    if wl.kind != "sat":
        cfg["result"] = {k: v for k, v in r["result"].items() if k not in ("device_ms", "wall_ms")}
    cfg["parallelism"] = ("index space split over %d GPU(s)" % world) if wl.kind == "sat" else \
        "replica per GPU (%d)" % world
    cfg["l2"] = ("no memory inputs (assignments come from thread indices); " if wl.kind != "stop" else
                 "table rebuilt every step; ") + "256 MB written between steps to flush L2"
    line = {
        "metric": wl.metric, "value": value, "unit": wl.metric, "n_gpus": world, "steps": steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "strong" if wl.kind == "sat" else "weak", "vs_baseline": None,
        "dtype": "u32 bit-sliced (lop3.b32)" if wl.kind != "stop" else "u32/u64 table entries",
        "data": "synthetic", "config": cfg,
        "roofline": wl.roofline(world, ms_step, peak_lop3, probe_mhz),
        "cpu_baseline": cpu,
        "e2e": {"value": e2e, "unit": wl.metric, "h2d_bytes_per_step": int(32 * lps),
                "d2h_bytes_per_step": int(32 * lps)},
        "e2e_cold": cold,
        "gpu_launches": launches,
        "clocks": clk,
        "warmup_s": t_warm,
    }
    if wl.kind == "sat":
        # the metric counts every gate of the circuit; the evaluator runs the
        # live ones (those the output depends on), covered by fewer LUTs
        line["live_gate_evals_per_s"] = value * wl.live / wl.circ.num_gates
        line["live_gates"] = wl.live
    print(json.dumps(line), flush=True)


def cold_probe(args, local):
    """The first solve of the workload in a new process with an empty kernel
    cache: context creation, LUT mapping, source generation, NVRTC compile,
    module load, launches and readback.  Returns its timings (or None)."""
    tmp = tempfile.mkdtemp(prefix="nsat_cold_")
    # empty kernel caches: this library's and the CUDA compute cache, where
    # NVRTC also keeps what it compiled
    env = dict(os.environ, NSAT_JIT_CACHE=tmp, CUDA_CACHE_PATH=os.path.join(tmp, "cuda"))
    cmd = [sys.executable, os.path.abspath(__file__), "--cold-probe", "--workload", args.workload,
           "--log2", str(args.log2), "--device", str(local)]
    try:
        out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=600)
        for line in out.stdout.splitlines()[::-1]:
            if line.startswith("{"):
                d = json.loads(line)
                d["note"] = ("first solve in a new process with an empty kernel cache (NVRTC compile and "
                             "module load included); context creation reported apart")
                return d
    except Exception:
        pass
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
    return None


def run_cold_probe(args):
    from naivesat_b200 import api
    wl = make_workload(args.workload, args.log2)
    t0 = time.perf_counter()
    ctx = api.Context(args.device)
    t1 = time.perf_counter()
    wl.setup(ctx, 1, 0)
    r = wl.step(fresh=False)
    t2 = time.perf_counter()
    print(json.dumps({"context_ms": 1e3 * (t1 - t0), "solve_ms": 1e3 * (t2 - t1),
                      "device_ms": r["device_ms"]}), flush=True)
    ctx.close()


# --------------------------------------------------------------------------
# config 4: batched serving

def replay_probe(args, local, count, srv_kw, realtime=True, mode="replay", repeat=1):
    """Runs one serving form over the first `count` requests of the trace in a
    new process with empty kernel caches (this library's and the CUDA compute
    cache).  Every request of the trace is a different circuit, so a server
    in service compiles each QSAT tiering kernel once; replaying the same
    requests in one process would find the kernels that an earlier replay
    compiled.  mode "replay": the batched server (all requests at t=0, or at
    their arrival times when realtime); mode "alone": one request at a time
    through a server holding no other job.  With repeat=2 the same form runs
    a second time in the same process (every kernel cached).  Returns the
    child's JSON: per run the verdicts, compiled blocks, latencies, makespan
    and server counters."""
    tmp = tempfile.mkdtemp(prefix="nsat_replay_")
    env = dict(os.environ, NSAT_JIT_CACHE=tmp, CUDA_CACHE_PATH=os.path.join(tmp, "cuda"))
    spec = {"count": count, "realtime": realtime, "srv_kw": srv_kw, "mode": mode, "repeat": repeat,
            "requests": args.requests, "rate": args.rate}
    cmd = [sys.executable, os.path.abspath(__file__), "--replay-probe", json.dumps(spec), "--device", str(local)]
    try:
        out = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=1800)
        for line in out.stdout.splitlines()[::-1]:
            if line.startswith("{"):
                return json.loads(line)
        raise RuntimeError("replay probe printed no result: " + out.stderr[-2000:])
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def run_replay_probe(args):
    from naivesat_b200 import api, serving, workloads as W
    spec = json.loads(args.replay_probe)
    ctx = api.Context(args.device)
    reqs = W.serving_requests(spec["requests"], seed=2024, rate_hz=spec["rate"])[:spec["count"]]
    warm = W.serving_requests(64, seed=99, rate_hz=1e9)
    kw = spec["srv_kw"]
    srv = api.Server(ctx, **kw)
    serving.replay_server(srv, warm, realtime=False)      # graphs captured, context warm
    srv.close()
    runs = []
    for _ in range(spec["repeat"]):
        srv = api.Server(ctx, **kw)
        if spec["mode"] == "alone":
            res, service = serving.interpreter_alone_service_times(srv, reqs)
            lat, mk = service, sum(service)
        else:
            res, lat, mk = serving.replay_server(srv, reqs, realtime=spec["realtime"])
        st = srv.stats()
        srv.close()
        keys = sorted(res)
        runs.append({"verdicts": [list(serving.verdict(reqs[k]["kind"], res[k])) for k in keys],
                     "compiled_blocks": [res[k]["compiled_blocks"] for k in keys],
                     "tiles": [res[k]["tiles"] for k in keys],
                     "lat": lat, "makespan": mk, "epochs": st["epochs"], "device_ms": st["device_ms"],
                     "shape": st["shape"]})
    print(json.dumps({"runs": runs}), flush=True)
    ctx.close()


def serving_cpu_baseline(reqs, threads, target_s):
    """The oracle port solving requests in order on the host cores for about
    target_s seconds; returns (solves/s, sample description)."""
    from oracle import oracle as O
    t0 = time.perf_counter()
    k = 0
    for r in reqs:
        if time.perf_counter() - t0 > target_s:
            break
        c = r["circ"]
        oc = O.Circuit(c.n, c.gates, c.outputs)
        if r["kind"] == "sat":
            # growing chunks, ending at the first chunk with a solution (the
            # lowest witness, as the server reports it)
            b, span = 0, 1 << min(c.n, 20)
            while b < (1 << c.n):
                e = min(1 << c.n, b + span)
                if O.sat_range(oc, b, e, threads)[1] is not None:
                    break
                b, span = e, span * 2
        elif r["kind"] == "qsat":
            O.qsat(oc, r["quants"], mode=1, threads=threads)
        else:
            O.stop_solve(c.n, r["unknowns"], O.stop_table(oc, threads), mode=1, threads=threads)
        k += 1
    dt = time.perf_counter() - t0
    return k / dt, "first %d requests of the trace in %.1f s" % (k, dt)


def run_serving_reference(args, world, rank):
    """Reference arm of config 4: the oracle port of the reference's CPU path
    solving the trace's requests one after another on all host cores (the
    reference runs one circuit per process and has no server)."""
    if rank != 0:
        return
    from naivesat_b200 import workloads as W
    reqs = W.serving_requests(args.requests, seed=2024, rate_hz=args.rate)
    threads = os.cpu_count() or 1
    vals = []
    for _ in range(max(1, args.steps)):
        v, sample = serving_cpu_baseline(reqs, threads, 20.0)
        vals.append(v)
    v = statistics.median(vals)
    line = {"impl": "reference", "metric": "solves/s", "value": v, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": 0, "ms_per_step": 1e3 / v, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u64 bit-sliced", "data": "synthetic",
            "config": {"workload": "config 4 trace, requests solved in order on the host", "cpu": cpu_model()},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": threads, "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def sm_count(device):
    import torch
    return torch.cuda.get_device_properties(device).multi_processor_count


def run_serving(args, world, rank, local):
    """Config 4: 10,000 SAT/QSAT/SATOSTOP requests (70/20/10) with Poisson
    arrivals through the batched server, against the plain one-launch-per-
    instance form on the same trace."""
    if rank != 0:
        return        # one server per GPU; the trace is served on rank 0's GPU
    from naivesat_b200 import api, serving, workloads as W
    ctx = api.Context(local)
    reqs = W.serving_requests(args.requests, seed=2024, rate_hz=args.rate)
    warm = W.serving_requests(64, seed=99, rate_hz=1e9)
    # the interpreter's shape and epoch budget for this GPU (persisted in the
    # kernel cache; servers created with the defaults use them)
    if args.shape:
        tune = {"shape": args.shape, "note": "given on the command line, not tuned"}
        srv_kw = dict(shape=args.shape)
    else:
        tune = api.server_tune(ctx, persist=True, retune=True)
        srv_kw = dict()
    if args.epoch_budget:
        srv_kw["epoch_budget"] = args.epoch_budget
    if args.rollover:
        srv_kw["rollover"] = True
    if args.max_slice_tiles:
        srv_kw["max_slice_tiles"] = args.max_slice_tiles
    if args.tier_min_ms:
        srv_kw["tier_min_ms"] = args.tier_min_ms
    if args.first_slice_tiles:
        srv_kw["first_slice_tiles"] = args.first_slice_tiles
    if args.tier_threads:
        srv_kw["tier_threads"] = args.tier_threads

    # every server of this run (here and in the fresh processes below) with the
    # same explicit shape and budget
    srv_kw.setdefault("shape", tune["shape"])
    srv_kw.setdefault("epoch_budget", tune.get("epoch_budget") or 12000000)

    peak_lop3, probe_mhz = ctx.lop3_peak()
    srv = api.Server(ctx, **srv_kw)
    serving.replay_server(srv, warm, realtime=False)      # graphs captured, context warm
    srv.close()

    # the saturated run: the first replay of the trace in this process, so its
    # QSAT tiering compiles every kernel it uses
    clocks = ClockSampler(local)
    clocks.start()
    srv = api.Server(ctx, **srv_kw)
    res_sat, lat_sat, mk_sat = serving.replay_server(srv, reqs, realtime=False)
    st_sat = srv.stats()
    srv.close()
    clk = clocks.stop()
    # the Poisson run in a new process with empty kernel caches: a replay here
    # would find the tiering kernels the saturated run compiled
    poi = replay_probe(args, local, len(reqs), srv_kw, realtime=True)["runs"][0]
    lat_poi, mk_poi = poi["lat"], poi["makespan"]
    st_poi = {"epochs": poi["epochs"]}
    for i in res_sat:
        assert tuple(poi["verdicts"][i]) == serving.verdict(reqs[i]["kind"], res_sat[i]), i

    # the plain forms, one request at a time, on the first kp requests of the
    # trace (kp: what the compile-bound form gets through in plain_seconds):
    # compiled one-shot solvers with an empty kernel cache (a new process per
    # circuit) and the same with every kernel already in the on-disk cache; the
    # precompiled interpreter serving one job at a time (no batching) and the
    # batched server on the same requests, each in a new process with empty
    # kernel caches, and the server once more with its kernels cached
    cache_dir = tempfile.mkdtemp(prefix="nsat_plain_")
    try:
        pres, service = serving.plain_service_times(ctx, reqs, args.plain_seconds, cache_dir=cache_dir)
        kp = len(service)
        prefix = reqs[:kp]
        wres, wservice = serving.plain_service_times(ctx, prefix, 1e9, cache_dir=cache_dir)
    finally:
        shutil.rmtree(cache_dir, ignore_errors=True)
    alone = replay_probe(args, local, kp, srv_kw, mode="alone")["runs"][0]
    iservice = alone["lat"]
    bsat = replay_probe(args, local, kp, srv_kw, realtime=False, repeat=2)["runs"]
    bpoi = replay_probe(args, local, kp, srv_kw, realtime=True, repeat=2)["runs"]
    same = 0
    for i in range(kp):
        v = serving.verdict(reqs[i]["kind"], res_sat[i])
        forms = [serving.verdict(reqs[i]["kind"], f) for f in (pres[i], wres[i])] + \
                [tuple(r["verdicts"][i]) for r in [alone] + bsat + bpoi]
        assert all(f == v for f in forms), i
        same += 1
    arr = [r["arrival_s"] for r in prefix]
    server_prefix = serving.summarize(bpoi[0]["lat"], bpoi[0]["makespan"], kp)
    server_prefix["solves_per_s"] = kp / bsat[0]["makespan"]
    server_prefix["note"] = ("a new process with empty kernel caches: solves/s with the requests queued at t=0, "
                             "latencies under the Poisson arrivals")
    server_warm = serving.summarize(bpoi[1]["lat"], bpoi[1]["makespan"], kp)
    server_warm["solves_per_s"] = kp / bsat[1]["makespan"]
    server_warm["note"] = ("the same server replaying the requests a second time in that process, every QSAT "
                           "tiering kernel cached: the like-for-like partner of the warm compiled form")

    def one_at_a_time(svc, form):
        lat = serving.fifo_latencies(arr, svc)
        sps = kp / sum(svc)
        return {"form": form, "solves_per_s": sps,
                "p50_ms_at_rate": serving.percentile(lat, 50) * 1e3,
                "p99_ms_at_rate": serving.percentile(lat, 99) * 1e3,
                "service_p50_ms": serving.percentile(svc, 50) * 1e3,
                "service_p99_ms": serving.percentile(svc, 99) * 1e3,
                "server_speedup": server_prefix["solves_per_s"] / sps,
                "warm_server_speedup": server_warm["solves_per_s"] / sps,
                "keeps_up_at_rate": sps > args.rate}
    plain_forms = {
        "requests": kp, "rate_hz": args.rate, "server": server_prefix, "server_warm_cache": server_warm,
        "interpreter_alone": one_at_a_time(iservice, "the precompiled interpreter, one job per server at a "
                                                     "time (same server options, no batching), in a new "
                                                     "process with empty kernel caches"),
        "compiled_warm_cache": one_at_a_time(wservice, "one-shot solvers with every kernel already in the "
                                                       "on-disk cache (a second pass over the same requests)"),
        "compiled_cold_cache": one_at_a_time(service, "one-shot solvers with an empty kernel cache (per-circuit "
                                                      "NVRTC compile, as one new process per circuit)"),
        "latency_note": "one-at-a-time forms: FIFO latencies from their measured service times under the same "
                        "arrivals; the server: measured under those arrivals",
        "verdicts_equal": same,
    }

    # a rate the plain form sustains: both forms on the same arrivals
    low = W.serving_requests(max(8, int(args.low_rate * args.low_seconds)), seed=77, rate_hz=args.low_rate)
    srv = api.Server(ctx, **srv_kw)
    res_low, lat_low, mk_low = serving.replay_server(srv, low, realtime=True)
    srv.close()
    pres_low, svc_low = serving.plain_service_times(ctx, low, 1e9)
    assert all(serving.verdict(low[i]["kind"], pres_low[i]) == serving.verdict(low[i]["kind"], res_low[i])
               for i in pres_low)
    plain_low_lat = serving.fifo_latencies([r["arrival_s"] for r in low], svc_low)

    # interpreter work: tiles x LUTs x 1024 words per tile (padding NOPs not counted)
    shape = st_sat["shape"]
    from concurrent.futures import ThreadPoolExecutor
    with ThreadPoolExecutor(max_workers=os.cpu_count() or 4) as pool:    # the ABI call releases the GIL
        luts = list(pool.map(lambda r: api.server_program_check(r["circ"], r["kind"], shape=shape)[1], reqs))
    words = sum(res_sat[i]["tiles"] * 1024 * luts[i] for i in res_sat)
    lut_words = words / (st_sat["device_ms"] * 1e-3)
    # every LUT-word reads three slot words and writes one in shared memory:
    # 16 bytes against 128 bytes per SM clock
    smem_peak = sm_count(local) * 128 * probe_mhz * 1e6 / 1e9
    cpu = None
    if not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        v, sample = serving_cpu_baseline(reqs, threads, 15.0)
        cpu = {"value": v, "unit": "solves/s", "cores": threads, "kind": "port", "sample": sample + ", " + cpu_model()}
    kinds = {k: sum(1 for r in reqs if r["kind"] == k) for k in ("sat", "qsat", "stop")}
    sat_sum = serving.summarize(lat_sat, mk_sat, len(res_sat))
    poi_sum = serving.summarize(lat_poi, mk_poi, len(lat_poi))
    poi_sum["note"] = "a new process with empty kernel caches (QSAT tiering compiles its kernels during the run)"
    # where the tail comes from: percentiles per kind, and for the QSAT jobs
    # that raced a compiled kernel
    groups = {}
    for k, lat in enumerate(lat_poi):
        groups.setdefault(reqs[k]["kind"], []).append(lat)
        if poi["compiled_blocks"][k]:
            groups.setdefault("qsat_tiered", []).append(lat)
    poi_sum["by_kind"] = {g: {"requests": len(v), "p50_ms": serving.percentile(v, 50) * 1e3,
                              "p99_ms": serving.percentile(v, 99) * 1e3} for g, v in groups.items()}
    line = {
        "metric": "solves/s", "value": sat_sum["solves_per_s"], "unit": "solves/s", "n_gpus": 1,
        "steps": len(reqs), "warmup": len(warm), "ms_per_step": 1e3 / sat_sum["solves_per_s"],
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "u32 bit-sliced (lop3.b32 LUT interpreter)", "data": "synthetic",
        "config": {"workload": "config 4: %d requests (%d SAT, %d QSAT, %d SATOSTOP), 18-34 inputs, 100-4000 "
                               "gates (log-uniform), SATOSTOP <= 20 state bits; server with all requests queued "
                               "at t=0 (value) and with Poisson arrivals at %.0f/s (latency)"
                               % (len(reqs), kinds["sat"], kinds["qsat"], kinds["stop"], args.rate),
                   "step": "one request solved", "epochs": st_sat["epochs"],
                   "server_options": {k: (bool(v) if k == "rollover" else v) for k, v in srv_kw.items()},
                   "qsat_tiering": {"jobs": sum(1 for r in res_sat.values() if r["compiled_blocks"]),
                                    "compiled_blocks": sum(r["compiled_blocks"] for r in res_sat.values()),
                                    "note": "large QSAT jobs race a kernel compiled for them; its 1/16 prefix "
                                            "blocks take over once it is ready"},
                   "l2": "no memory inputs (assignments come from thread indices)"},
        "latency": dict(poi_sum, rate_hz=args.rate, epochs=st_poi["epochs"]),
        "plain_forms": plain_forms,
        "low_rate": {"rate_hz": args.low_rate, "requests": len(low),
                     "server": serving.summarize(lat_low, mk_low, len(res_low)),
                     "plain": serving.summarize(plain_low_lat, sum(svc_low), len(svc_low))},
        "roofline": {"bound": "smem", "kernel": "serve_epoch",
                     "achieved": lut_words * 16 / 1e9, "peak": smem_peak, "unit": "GB/s",
                     "frac": lut_words * 16 / 1e9 / smem_peak, "traffic": None,
                     "lut_words_per_s": lut_words, "lop3_issue_frac": lut_words / peak_lop3,
                     "note": "each LUT-word reads 3 and writes 1 slot word of shared memory (16 B); peak = SMs x "
                             "128 B/clk x the SM clock the lop3 probe measured",
                     "peak_source": "architectural shared-memory width x measured clock (%.0f MHz)" % probe_mhz},
        "interpreter_tuning": dict(tune, shape_used=shape),
        "cpu_baseline": cpu,
        "e2e": {"value": sat_sum["solves_per_s"], "unit": "solves/s",
                "h2d_bytes_per_step": st_sat["h2d_bytes"] / len(reqs),
                "d2h_bytes_per_step": st_sat["d2h_bytes"] / len(reqs),
                "note": "the server runs end to end: circuits arrive as host arrays, programs and epoch tables "
                        "are copied in, results copied out; bytes per request from the server's counters"},
        # interpreter epochs and join rounds, plus at least one launch per compiled block
        "gpu_launches": st_sat["launches"] + sum(r["compiled_blocks"] for r in res_sat.values()),
        "clocks": clk,
    }
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="c1")
    ap.add_argument("--log2", type=int, default=36,
                    help="SAT workloads: enumerate only the first 2^LOG2 assignments (profiling)")
    ap.add_argument("--no-cpu-baseline", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--requests", type=int, default=10000, help="c4: requests in the trace")
    ap.add_argument("--rate", type=float, default=150.0, help="c4: Poisson arrival rate (1/s)")
    ap.add_argument("--plain-seconds", type=float, default=60.0, help="c4: time given to the plain form")
    ap.add_argument("--low-rate", type=float, default=2.0, help="c4: a rate the plain form sustains")
    ap.add_argument("--low-seconds", type=float, default=45.0, help="c4: length of the low-rate trace")
    ap.add_argument("--no-e2e-cold", action="store_true", help="skip the cold-start (new process) solve")
    ap.add_argument("--shape", type=int, default=0, help="c4: interpreter shape 1..6 instead of tuning one")
    ap.add_argument("--epoch-budget", type=int, default=0, help="c4: epoch budget instead of the tuned one")
    ap.add_argument("--rollover", action="store_true", help="c4: servers with roll-over into the next slices")
    ap.add_argument("--max-slice-tiles", type=int, default=0, help="c4: largest slice of a job per epoch (tiles)")
    ap.add_argument("--tier-min-ms", type=int, default=0, help="c4: QSAT jobs estimated above this race a compiled kernel")
    ap.add_argument("--first-slice-tiles", type=int, default=0, help="c4: a new job's first slice (tiles)")
    ap.add_argument("--tier-threads", type=int, default=0, help="c4: QSAT tiering workers")
    ap.add_argument("--cold-probe", action="store_true", help=argparse.SUPPRESS)
    ap.add_argument("--replay-probe", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--device", type=int, default=0, help=argparse.SUPPRESS)
    args = ap.parse_args()
    if args.cold_probe:
        run_cold_probe(args)
        return
    if args.replay_probe:
        run_replay_probe(args)
        return
    # NVRTC keeps compiled kernels in the CUDA compute cache (CUDA_CACHE_PATH,
    # by default shared by every process of the user), so a kernel that an
    # earlier run compiled would make this run's cold figures (e2e_cold, the
    # empty-cache plain form of c4) warm.  Every run starts from an empty one.
    cuda_cache = tempfile.mkdtemp(prefix="nsat_cuda_cache_")
    os.environ["CUDA_CACHE_PATH"] = cuda_cache
    try:
        run_main(args)
    finally:
        shutil.rmtree(cuda_cache, ignore_errors=True)


def run_main(args):
    world, rank, local = dist_setup()
    try:
        if args.workload == "c4":
            if args.impl == "reference":
                run_serving_reference(args, world, rank)
            else:
                run_serving(args, world, rank, local)
        elif args.impl == "reference":
            run_reference(args, world, rank)
        else:
            run_ours(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

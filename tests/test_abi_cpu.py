"""Host-side checks that need no GPU: the C ABI loads and exports every
declared symbol, text I/O round-trips, and every kernel kind NVRTC-compiles
for sm_100a."""
import os
import re

import pytest

from naivesat_b200 import api
from naivesat_b200 import workloads as W

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    text = open(os.path.join(ROOT, "include", "nsat.h")).read()
    text = re.sub(r"/\*.*?\*/", "", text, flags=re.S)
    return sorted(set(re.findall(r"\b(nsat_[a-z0-9_]+)\s*\(", text)))


def test_library_exports_every_declared_symbol():
    L = api.lib()
    syms = declared_symbols()
    assert len(syms) >= 20
    for s in syms:
        assert hasattr(L, s), s
    assert set(api.EXPORTS) <= set(syms)


def test_no_device_is_reported_cleanly():
    if api.device_count() > 0:
        pytest.skip("a device is present")
    with pytest.raises(api.NsatError, match="no CUDA device"):
        api.Context(0)


def test_strerror_codes():
    L = api.lib()
    for code in range(-9, 1):
        assert L.nsat_strerror(code)


def test_gatesim_text_roundtrip():
    for name in ["c0", "c2a", "c3b"]:
        c = W.config(name)
        text = api.format_circuit(c.n, c.gates, c.outputs, c.quants)
        n, gates, outs, quants = api.parse(text)
        assert n == c.n
        assert (gates == c.gates).all() and (outs == c.outputs).all()
        assert quants == c.quants


def test_gatesim_text_examples():
    n, g, o, q = api.parse("{0 1 2 and(0,1) nor(2,3):0n xor(3,4):1}(3)")
    assert n == 3 and g.tolist() == [[0, 0, 1], [1, 2, 3], [3, 3, 4]]
    assert o.tolist() == [[4, 1], [5, 0]] and q is None
    n, g, o, q = api.parse("ae a {0 1 2 nimpl(0,1):0}(3)")
    assert q == "AEA" and g.tolist() == [[2, 0, 1]]
    n, g, o, q = api.parse("{0:0 1:1n}(2)")     # identity outputs on inputs
    assert o.tolist() == [[0, 0], [1, 1]]
    for bad in ["{0 1 and(0,5):0}(2)", "{0 1 foo(0,1):0}(2)", "{0 1 and(0,1)}(2)", "{0:1}(1)"]:
        with pytest.raises(api.NsatError):
            api.parse(bad)


def test_negation_folding_preserves_function():
    """The generators fold negated fan-ins into gatesim gates; the folded
    circuit must compute what the raw gates describe."""
    rng = W.SplitMix64(5)
    for t in range(20):
        n = 6
        rb = W.random_dag_raw(rng, n, 40, window=8)
        rb.output(n + 39)
        rb.output(n + 20, 1)
        c = rb.fold()
        for v in range(1 << n):
            bits = [(v >> i) & 1 for i in range(n)]
            w = bits + [0] * len(rb.raw)
            for k, (f, a, na, b, nb) in enumerate(rb.raw):
                w[n + k] = W._gate(f, w[a] ^ na, w[b] ^ nb)
            exp = [w[n + 39], w[n + 20] ^ 1]
            assert c.eval_bits(bits) == exp


@pytest.mark.parametrize("name,kind", [("c0", "sat"), ("c2a", "qsat"), ("c3b", "table"),
                                       ("c3a", "table")])
def test_kernels_compile_for_sm100a(name, kind):
    c = W.config(name)
    r = api.jit_check(c, kind, quants=c.quants)
    assert r["regs"] > 0, r["log"]
    assert r["spill_bytes"] == 0, r["log"]
    assert r["lop3_ops"] <= r["live_gates"]


def test_one_op_per_gate_mode_compiles():
    c = W.config("c0")
    r = api.jit_check(c, "sat", no_optimize=True)
    assert r["lop3_ops"] == r["live_gates"]


def test_lut_mapping_saves_ops():
    c = W.config("c1")
    fused = api.jit_check(c, "sat")
    assert fused["lop3_ops"] < 0.8 * fused["live_gates"], fused


@pytest.mark.parametrize("name,kind,lop3", [("c0", "sat", 280), ("c1", "sat", 1229), ("c1_twin", "sat", 1354),
                                            ("c2a", "qsat", 38), ("c2c", "qsat", 665)])
def test_lut_counts_of_the_benchmark_circuits(name, kind, lop3):
    """The mapper is deterministic; these covers are the ones the measured
    rooflines count.  c0's 2^24 search is short next to cut mapping, so its
    cover is one LUT per live gate (280); the others are cut covers."""
    c = W.config(name)
    assert api.jit_check(c, kind, quants=c.quants)["lop3_ops"] == lop3


@pytest.mark.parametrize("seed,n,g,out", [(0, 24, 500, "last"), (1, 36, 3000, "live"), (3, 30, 1500, "live"),
                                          (77, 18, 100, "last"), (123456789, 34, 4000, "live")])
def test_library_generator_matches_python(seed, n, g, out):
    a = W.random_dag(seed, n, g, output=out)
    b = W.random_dag_py(seed, n, g, output=out)
    assert (a.gates == b.gates).all() and (a.outputs == b.outputs).all()


@pytest.mark.parametrize("seed,n,g", [(4, 24, 300), (4, 32, 300), (99, 15, 120)])
def test_library_lfsr_generator_matches_python(seed, n, g):
    a = W.lfsr_stop(seed, n, g)
    b = W.lfsr_stop_py(seed, n, g)
    assert (a.gates == b.gates).all() and (a.outputs == b.outputs).all() and a.pattern == b.pattern


@pytest.mark.parametrize("seed,n,g", [(1, 34, 4000), (2, 30, 1000), (3, 20, 100), (4, 26, 600), (9, 18, 60),
                                      (11, 22, 2500)])
def test_server_program_matches_circuit(seed, n, g):
    """The interpreter program (groups of independent LUTs, recycled slots)
    computes the circuit's output on random assignments."""
    c = W.random_dag(seed, n, g, output="live")
    slots, luts, nops = api.server_program_check(c, "sat", seed=seed)
    assert luts > 0 and slots <= 384
    assert nops <= luts // 4 + 8


@pytest.mark.parametrize("shape", range(1, api.SERVE_SHAPES + 1))
def test_server_programs_of_every_shape(shape):
    """Every interpreter shape's group size gives a program that computes the
    circuit (groups of 1, 2 or 4 independent instructions)."""
    for seed, n, g in [(1, 34, 4000), (4, 26, 600), (9, 18, 60)]:
        c = W.random_dag(seed, n, g, output="live")
        slots, luts, nops = api.server_program_check(c, "sat", seed=seed, shape=shape)
        assert slots <= 384 and luts > 0
    api.server_program_check(W.config("c3a"), "stop", shape=shape)


def test_server_program_check_on_config_circuits():
    for name, kind in [("c0", "sat"), ("c1", "sat"), ("c2a", "qsat"), ("c2c", "qsat"), ("c3a", "stop"),
                       ("c3b", "stop")]:
        api.server_program_check(W.config(name), kind)
    for r in W.serving_requests(60, seed=3, rate_hz=1e9, n_range=(12, 22), g_range=(40, 900),
                                stop_n_range=(8, 14)):
        api.server_program_check(r["circ"], r["kind"], seed=5)


def test_lru_map_matches_model(tmp_path):
    """The bounded map behind the in-memory kernel cache agrees with a plain
    model on random finds, puts, replacements and capacity changes."""
    import shutil
    import subprocess
    if shutil.which("g++") is None:
        pytest.skip("g++ not available")
    here = os.path.dirname(os.path.abspath(__file__))
    exe = str(tmp_path / "lru_check")
    subprocess.run(["g++", "-O1", "-std=c++17", "-I", os.path.join(here, "..", "naivesat_b200", "csrc"),
                    os.path.join(here, "lru_check.cpp"), "-o", exe], check=True)
    r = subprocess.run([exe], capture_output=True, text=True, timeout=120)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr


def test_short_search_cover_rule_is_for_solves_that_own_the_device():
    """c0's 2^24 search is short next to cut mapping: a one-shot solve takes
    one LUT per live gate (280), while the same circuit served (its device
    time shared by every job) keeps the 170-LUT cut cover."""
    c = W.config("c0")
    assert api.jit_check(c, "sat")["lop3_ops"] == 280
    assert api.server_program_check(c, "sat")[1] == 170

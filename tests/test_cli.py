"""The four command-line tools: argument handling (CPU) and end-to-end
answers on circuit files (GPU), in the reference's output formats."""
import os
import subprocess

import pytest

from naivesat_b200 import api
from naivesat_b200 import workloads as W
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "naivesat_b200", "bin")
TOOLS = ["naivesat", "naiveqsat", "naivesatostop", "greedysatostop"]


def run(tool, *args, check=False, env=None):
    p = subprocess.run([os.path.join(BIN, tool)] + [str(a) for a in args], capture_output=True,
                       text=True, timeout=600, env=dict(os.environ, **env) if env else None)
    if check:
        assert p.returncode == 0, p.stdout + p.stderr
    return p


def write(tmp_path, circ, name):
    path = tmp_path / (name + ".circuit")
    path.write_text(api.format_circuit(circ.n, circ.gates, circ.outputs, circ.quants))
    return path


@pytest.mark.parametrize("tool", TOOLS)
def test_help_and_bad_args(tool):
    p = run(tool, "--help")
    assert p.returncode == 0 and "Usage:" in p.stdout
    p = run(tool, "--bogus-flag", "x")
    assert p.returncode == 2
    p = run(tool, "/nonexistent.circuit", "3", "-t", "opencl:0")
    assert p.returncode != 0


def test_exec_type_is_required(tmp_path):
    path = write(tmp_path, W.config("c0"), "c0")
    p = run("naivesat", path)
    assert p.returncode == 2 and "exec-type" in p.stderr


gpu = pytest.mark.gpu


def bits(v, n):
    return format(v, "0%db" % n)


@gpu
def test_naivesat_cli(tmp_path):
    c = W.config("c0")
    cnt, low = O.sat_range(O.Circuit(c.n, c.gates, c.outputs))
    out = run("naivesat", write(tmp_path, c, "c0"), "-t", "opencl:0", check=True).stdout
    assert "Found Input: %s\n" % bits(low, c.n) in out
    out = run("naivesat", write(tmp_path, c, "c0"), "-t", "cpu_and_opencl", "-e", "20", check=True).stdout
    assert "Found Input: %s\n" % bits(low, c.n) in out
    unsat = W.Circuit(16, [(W.NIMPL, 3, 3)], [(16, 0)])
    out = run("naivesat", write(tmp_path, unsat, "u"), "-t", "opencl:0", check=True).stdout
    assert out.rstrip().endswith("Unsatisfiable!")
    small = W.random_dag(3, 10, 40, output="live")
    cnt, low = O.sat_range(O.Circuit(small.n, small.gates, small.outputs))
    out = run("naivesat", write(tmp_path, small, "s"), "-t", "opencl:0", check=True).stdout
    assert ("Found Input: %s\n" % bits(low, 10)) in out if low is not None else "Unsatisfiable!" in out


@gpu
def test_naiveqsat_cli(tmp_path):
    out = run("naiveqsat", write(tmp_path, W.config("c2a"), "a"), "-t", "opencl:0", check=True).stdout
    assert "Result: (Satisfiable)\n" in out
    out = run("naiveqsat", write(tmp_path, W.config("c2b"), "b"), "-t", "opencl:0", check=True).stdout
    assert "Result: (Unsatisfiable: %s)\n" % ("0" * 16) in out
    # plain circuit: every input existential (qsat.rs:6277-6285)
    c = W.random_dag(5, 16, 120, output="live")
    exp = O.qsat(O.Circuit(c.n, c.gates, c.outputs), "E" * 16)
    out = run("naiveqsat", write(tmp_path, c, "p"), "-t", "cpu", check=True).stdout
    if exp["solution"] is None:
        assert "Result: (Unsatisfiable)\n" in out
    else:
        assert "Result: (Satisfiable: %s)\n" % bits(exp["solution"], 16) in out


@gpu
def test_satostop_clis(tmp_path):
    path = write(tmp_path, W.config("c3b"), "cnt")
    out = run("greedysatostop", path, 16, "-v", check=True).stdout
    assert "Solution: Solution { start: 16776960, end: 0 }\n" in out
    assert "Verified: end=0\n" in out and "INCORRECT" not in out
    out = run("naivesatostop", path, 16, "-t", "opencl:0", "-v", check=True).stdout
    assert "Solution: Solution { start: 0, end: 0, steps: 16777216 }\n" in out
    assert "Verified: end=0 steps=16777216\n" in out and "INCORRECT" not in out
    # hashmap tuning flags of the reference's engine are accepted and change nothing
    out = run("naivesatostop", path, 16, "-t", "cpu", "-H", "20", "-U", "4", "-P", "2", "-C", "10",
              check=True).stdout
    assert "Solution: Solution { start: 0, end: 0, steps: 16777216 }\n" in out
    out = run("naivesatostop", path, 16, "-S", check=True).stdout
    assert "Stopped at %s %s\n" % ("0" * 16, "0" * 24) in out
    out = run("greedysatostop", write(tmp_path, W.config("c3a"), "lfsr"), 16, check=True).stdout
    assert "Unsatisfiable!" in out


@gpu
def test_greedy_partitions_cli(tmp_path):
    """greedysatostop -p P [-x PREFIX]: the reference's partitioned schedule."""
    c = W.lfsr_stop(5, 16, 48)
    path = write(tmp_path, c, "lfsr16")
    oc = O.Circuit(c.n, c.gates, c.outputs)
    exp = O.greedy_partitioned(16, 8, O.stop_table(oc), 4)
    spill = tmp_path / "spill"
    spill.mkdir()
    for extra in ([], ["-x", str(spill) + "/"]):
        out = run("greedysatostop", path, 8, "-p", "4", "-v", *extra, check=True).stdout
        assert "Load partition bits: 4\n" in out
        if exp is None:
            assert "Unsatisfiable!" in out
        else:
            assert "Solution: Solution { start: %d, end: %d }\n" % (exp["start"], exp["end"]) in out
            assert "INCORRECT" not in out
    assert list(spill.iterdir()) == []
    p = run("greedysatostop", path, 8, "-p", "3")
    assert p.returncode == 101 and "power of 2" in p.stderr + p.stdout


@gpu
def test_autotuned_clis_answer_the_same(tmp_path):
    """NSAT_AUTOTUNE=1 tunes the launch shape (kept in the kernel cache
    directory); the answer lines do not change."""
    env = {"NSAT_AUTOTUNE": "1", "NSAT_JIT_CACHE": str(tmp_path / "cache")}
    c = W.config("c0")
    path = write(tmp_path, c, "c0")
    plain = run("naivesat", path, "-t", "opencl:0", check=True).stdout
    tuned = run("naivesat", path, "-t", "opencl:0", check=True, env=env).stdout
    line = [x for x in plain.splitlines() if x.startswith(("Found Input", "Unsatisfiable"))]
    assert line and line[0] in tuned
    assert any(f.startswith("tune_") for f in os.listdir(tmp_path / "cache"))
    q = write(tmp_path, W.config("c2a"), "a")
    plain = run("naiveqsat", q, "-t", "opencl:0", check=True).stdout
    tuned = run("naiveqsat", q, "-t", "opencl:0", check=True, env=env).stdout
    res = [x for x in plain.splitlines() if x.startswith("Result:")]
    assert res and res[0] in tuned

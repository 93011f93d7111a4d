"""Parity at the full benchmark sizes, where the oracle would take hours:
size-independent properties of the CUDA path's answers.

- config 1, all 2^36 assignments: the count is the sum of the counts of four
  disjoint quarter ranges, the witness is the lowest of theirs, it satisfies
  the circuit on the CPU, it carries the planted block, and nothing below it
  is a solution (an empty device range up to its 1024-aligned floor, then
  the oracle over the last <= 1023 assignments).
- config 1 and its unplanted twin, all 2^36 assignments: the exact count and
  lowest witness equal those of the generated-code CPU path
  (oracle/cpu_codegen.py, itself pinned to the oracle's interpreter), an
  independent evaluator fast enough for the whole space (seconds on the
  host's cores).
- the 32-bit-state SATOSTOP scale-up (2^32 u64 entries): sampled table
  entries equal the oracle's next state and STOP, and the answer of the
  doubling is a start with its known bits zero whose run stops.
"""
import numpy as np
import pytest

from naivesat_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ["c1", "c1_twin"])
def test_full_count_matches_generated_cpu_path(ctx, name):
    from oracle import cpu_codegen as CG
    c = W.config(name)
    full = ctx.circuit(c).sat(find_all=True)
    g = CG.CodegenSat(c, 24)
    try:
        cnt, low = g.sat_args(0, 1 << (c.n - g.e))
    finally:
        g.close()
    assert (full["count"], full["witness"]) == (cnt, low), (name, full, cnt, low)


def test_config1_full_enumeration(ctx):
    c = W.config("c1")
    h = ctx.circuit(c)
    full = h.sat(find_all=True)
    q = 1 << 34
    parts = [h.sat(find_all=True, begin=k * q, end=(k + 1) * q) for k in range(4)]
    assert full["count"] == sum(p["count"] for p in parts)
    w = full["witness"]
    assert w == min(p["witness"] for p in parts if p["satisfiable"])
    oc = O.Circuit(c.n, c.gates, c.outputs)
    assert O.eval_scalar(oc, [(w >> i) & 1 for i in range(c.n)])[0] == 1
    assert w & ((1 << 18) - 1) == c.plant_k
    floor = w & ~1023
    assert w < (1 << 30)
    if floor:
        assert h.sat(find_all=True, begin=0, end=floor)["count"] == 0
    assert O.sat_range(oc, floor, w + 1)[1] == w
    first = h.sat(find_all=False)          # naivesat's stop-at-first mode
    assert first["satisfiable"] and first["witness"] == w


def test_scaleup_table_n32(ctx):
    c = W.lfsr_stop(4, 32, 300)
    n, u = 32, 20
    oc = O.Circuit(c.n, c.gates, c.outputs)
    h = ctx.circuit(c)
    t = h.stop_table()
    try:
        rng = np.random.default_rng(11)
        for s in [0, (1 << n) - 1] + [int(x) for x in rng.integers(0, 1 << n, 1024, dtype=np.uint64)]:
            out = O.eval_scalar(oc, [(s >> i) & 1 for i in range(n)])
            exp = sum(int(out[i]) << i for i in range(n)) | (int(out[n]) << n)
            assert int(t.read(s, 1)[0]) == exp, s
        r = t.solve(u, mode=0)
    finally:
        t.close()
    if r["found"]:
        assert r["start"] & ((1 << (n - u)) - 1) == 0
        rep = O.stop_replay(oc, r["start"], 1 << 22)
        if rep is not None:                # stops within 2^22 steps: the end must agree
            assert rep[0] == r["end"]

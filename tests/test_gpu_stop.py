"""SATOSTOP table build + pointer doubling (greedysatostop / naivesatostop
paths) against the oracle, through the C ABI."""
import numpy as np
import pytest

from naivesat_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def oc(c):
    return O.Circuit(c.n, c.gates, c.outputs)


@pytest.mark.parametrize("n", [3, 5, 8, 13, 20, 24])
def test_table_enumeration_layout(ctx, n):
    """Identity circuit: entry s = s | bit0(s) << n (the layout pin of
    satostop.rs:1789-1915, re-targeted at the next-state table)."""
    c = W.identity_stop(n, 0)
    t = ctx.circuit(c).stop_table()
    got = t.read()
    s = np.arange(1 << n, dtype=np.uint64)
    assert (got == (s | ((s & 1) << n))).all()


def test_table_matches_oracle(ctx):
    for name in ["c3a", "c3b"]:
        c = W.config(name)
        exp = O.stop_table(oc(c))
        got = ctx.circuit(c).stop_table().read()
        assert (got == exp).all(), name


def test_counter_known_answers(ctx):
    """Config 3b: every unknown start stops; the lowest overall is start 0
    (end 0, 2^24 steps); the first doubling round resolves start 0xFFFF00."""
    c = W.config("c3b")
    h = ctx.circuit(c)
    r1 = h.stop_table(want_steps=True).solve(16, mode=1)
    assert r1["found"] and (r1["start"], r1["end"], r1["steps"]) == (0, 0, 1 << 24)
    r0 = h.stop_table(want_steps=True).solve(16, mode=0)
    assert (r0["start"], r0["end"], r0["steps"], r0["rounds"]) == (0xFFFF00, 0, 256, 8)
    r = h.stop_table().solve(16, mode=0)
    assert (r["start"], r["end"], r["rounds"]) == (0xFFFF00, 0, 8)


@pytest.mark.parametrize("mode", [0, 1])
def test_lfsr_matches_oracle(ctx, mode):
    c = W.config("c3a")
    table = O.stop_table(oc(c))
    exp = O.stop_solve(24, 16, table, mode=mode)
    got = ctx.circuit(c).stop_table(want_steps=True).solve(16, mode=mode)
    if exp is None:
        assert not got["found"]
    else:
        assert got["found"] and (got["start"], got["end"], got["steps"], got["rounds"]) == \
            (exp["start"], exp["end"], exp["steps"], exp["rounds"])
        rep = O.stop_replay(oc(c), got["start"], 1 << 24)
        assert rep == (got["end"], got["steps"])


@pytest.mark.parametrize("seed", range(8))
def test_random_stop_circuits(ctx, seed):
    """Small random next-state circuits, both modes, both entry formats."""
    rng = W.SplitMix64(seed)
    n = 10 + seed
    u = max(1, n - 3 - rng.below(4))
    rb = W.random_dag_raw(rng, n, 6 * n, window=2 * n)
    last = n + 6 * n
    for i in range(n):
        rb.output(last - 1 - i)
    rb.output(rb.gate(W.AND, last - 1, last - 2))
    c = rb.fold()
    table = O.stop_table(oc(c))
    for mode in (0, 1):
        exp = O.stop_solve(n, u, table, mode=mode)
        for steps in (False, True):
            got = ctx.circuit(c).stop_table(want_steps=steps).solve(u, mode=mode)
            if exp is None:
                assert not got["found"]
                continue
            assert got["found"] and (got["start"], got["end"], got["rounds"]) == \
                (exp["start"], exp["end"], exp["rounds"])
            if steps:
                assert got["steps"] == exp["steps"]


def test_no_stop_anywhere(ctx):
    """check_stop: no state ever stops -> no solution, no rounds run."""
    n = 12
    rb = W.RawBuilder(n)
    z = rb.gate(W.NIMPL, 0, 0)       # constant 0
    for i in range(n):
        rb.output(i)
    rb.output(z)
    r = ctx.circuit(rb.fold()).stop_table().solve(n, mode=0)
    assert not r["found"] and r["rounds"] == 0


def test_repeated_tables_reuse_the_context_pool(ctx):
    """Tables come from the context's stream-ordered pool: building, solving
    and freeing the same 2^24-state table many times gives the same answer
    every time, and the device's free memory does not drift by more than
    the pool keeps for reuse (8 GiB) plus one table pair."""
    import torch
    c = W.config("c3a")
    h = ctx.circuit(c)
    free0 = torch.cuda.mem_get_info(0)[0]
    answers = set()
    for _ in range(12):
        t = h.stop_table()
        r = t.solve(12, mode=1)
        answers.add((r["found"], r.get("start"), r.get("end"), r["rounds"]))
        t.close()
    assert len(answers) == 1, answers
    free1 = torch.cuda.mem_get_info(0)[0]
    assert free0 - free1 <= (8 << 30) + 2 * (4 << 24), (free0, free1)

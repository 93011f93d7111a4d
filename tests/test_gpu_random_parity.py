"""Seeded random parity sweep: random circuits of random sizes, fan-in
windows and quantifier strings through every solver path (compiled SAT with
counts, compiled QSAT, full-table SATOSTOP in both modes, partitioned
greedysatostop with the image in device or pinned host memory) and through
one server that receives all of them, each against the oracle."""
import random

import pytest

from naivesat_b200 import api
from naivesat_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu


def test_random_parity_sweep(ctx):
    rng = random.Random(20261203)
    srv = api.Server(ctx)
    expected = {}
    for t in range(80):
        kind = rng.choice(["sat", "sat", "qsat", "stop"])
        seed = rng.randrange(1 << 30)
        if kind == "stop":
            n = rng.randrange(11, 16)
            c = W.lfsr_stop(seed, n, rng.randrange(n + 4, 100)) if rng.random() < 0.8 else W.counter_stop(n)
            oc = O.Circuit(c.n, c.gates, c.outputs)
            tab = O.stop_table(oc)
            u = rng.randrange(0, n + 1)
            for mode in (0, 1):
                exp = O.stop_solve(n, u, tab, mode=mode)
                tb = ctx.circuit(c).stop_table(want_steps=(mode == 1))
                got = tb.solve(u, mode=mode)
                tb.close()
                assert got["found"] == (exp is not None), (seed, n, u, mode)
                if exp is not None:
                    assert (got["start"], got["end"]) == (exp["start"], exp["end"]), (seed, n, u, mode)
                    if mode == 1:
                        assert got["steps"] == exp["steps"]
            P = rng.choice([2, 4, 8])
            exp = O.greedy_partitioned(n, u, tab, P)
            got = ctx.circuit(c).greedy_partitioned(u, P, device_bytes=rng.choice([0, 1]))
            assert got["found"] == (exp is not None), (seed, n, u, P)
            if exp is not None:
                assert (got["start"], got["end"]) == (exp["start"], exp["end"]), (seed, n, u, P)
            srv.submit("stop", c, unknowns=u, tag=t)
            expected[t] = ("stop", O.stop_solve(n, u, tab, mode=1))
            continue
        n = rng.randrange(6, 21)
        g = int(2 ** rng.uniform(2, 9))
        c = W.random_dag(seed, n, g, output=rng.choice(["live", "last"]), window=rng.choice([8, 16, 64]))
        oc = O.Circuit(c.n, c.gates, c.outputs)
        if kind == "sat":
            cnt, low = O.sat_range(oc)
            r = ctx.circuit(c).sat(find_all=True)
            assert (r["count"], r["witness"]) == (cnt, low), (seed, n, g)
            find_all = rng.random() < 0.5
            srv.submit("sat", c, tag=t, find_all=find_all)
            expected[t] = ("sat", (cnt if find_all else None, low))
        else:
            q = "".join(rng.choice("AE") for _ in range(n))
            e = O.qsat(oc, q, mode=1)
            r = ctx.circuit(c).qsat(q)
            ee = (e["reversed"], e["solution_bits"], e["solution"])
            assert (r["reversed"], r["solution_bits"], r["solution"]) == ee, (seed, n, g, q)
            srv.submit("qsat", c, quants=q, tag=t)
            expected[t] = ("qsat", ee)
    results = srv.run_all()
    assert len(results) == len(expected)
    for r in results:
        kind, exp = expected[r["tag"]]
        assert r["status"] == 0
        if kind == "sat":
            cnt, low = exp
            assert r["witness"] == low and (cnt is None or r["count"] == cnt), r
        elif kind == "qsat":
            assert (r["reversed"], r["solution_bits"], r["solution"]) == exp, r
        else:
            assert r["found"] == (exp is not None), r
            if exp is not None:
                assert (r["start"], r["end"], r["steps"]) == (exp["start"], exp["end"], exp["steps"]), r

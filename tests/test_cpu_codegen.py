"""The generated-code CPU baseline (oracle/cpu_codegen.py) gives the oracle's
count and lowest witness: config 0 in full and seeded random circuits over
several arg ranges (CPU only)."""
import pytest

from naivesat_b200 import workloads as W
from oracle import cpu_codegen as CG
from oracle import oracle as O


def check(circ, e, a0, a1):
    g = CG.CodegenSat(circ, e)
    try:
        got = g.sat_args(a0, a1)
        exp = O.sat_range(O.Circuit(circ.n, circ.gates, circ.outputs), a0 << g.e, a1 << g.e)
        assert got == exp, (circ.name, e, a0, a1, got, exp)
    finally:
        g.close()


def test_config0_in_full():
    c = W.config("c0")
    check(c, 20, 0, 1 << (c.n - 20))


@pytest.mark.parametrize("seed", range(6))
def test_random_circuits(seed):
    n = 14 + seed
    c = W.random_dag(300 + seed, n, 80 + 60 * seed, output="live")
    e = max(10, n - 3)
    check(c, e, 0, 1 << (n - e))
    check(c, e, 1, 3)


def test_negated_output_and_unsatisfiable():
    c = W.random_dag(7, 16, 200, output="live")
    w, neg = (int(x) for x in c.outputs[0])
    check(W.Circuit(c.n, c.gates, [(w, 1 - neg)], name="negated"), 12, 0, 16)
    # x0 AND NOT x0 (Nimpl x0, x0) has no solution
    check(W.Circuit(12, [(2, 0, 0)], [(12, 0)], name="contradiction"), 10, 0, 4)

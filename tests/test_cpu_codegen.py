"""The generated-code CPU baseline (oracle/cpu_codegen.py) gives the oracle's
count and lowest witness: config 0 in full and seeded random circuits over
several arg ranges; and its QSAT calls give the oracle's FinalResult, units
inside a call and units that span calls, with the adder formulas' known
answers (CPU only)."""
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


@pytest.mark.parametrize("seed", range(8))
def test_qsat_random_formulas(seed):
    import random
    rng = random.Random(40 + seed)
    n = (18, 20, 22)[seed % 3]
    c = W.random_dag(700 + seed, n, (60, 200, 500)[seed % 3], output="live")
    f = rng.randint(1, n - 9)
    q0 = rng.choice("AE")
    q = q0 * f + ("E" if q0 == "A" else "A") + "".join(rng.choice("AE") for _ in range(n - f - 1))
    exp = O.qsat(O.Circuit(c.n, c.gates, c.outputs), q, mode=1)
    for e in (None, 10, 12):          # whole units per call, and units over several calls
        g = CG.CodegenQsat(c, q, elem_bits=e)
        try:
            assert g.solve() == exp, (seed, q, e)
        finally:
            g.close()


def test_qsat_adder_known_answers():
    """config 2a is TRUE (no counterexample), config 2b FALSE with a = 0."""
    for name, exp in (("c2a", {"reversed": True, "solution_bits": 16, "solution": None}),
                      ("c2b", {"reversed": True, "solution_bits": 16, "solution": 0})):
        c = W.config(name)
        g = CG.CodegenQsat(c, c.quants)
        try:
            assert g.solve() == exp, name
        finally:
            g.close()


def test_qsat_units_below_a_vector_word_are_refused():
    c = W.random_dag(5, 16, 100, output="live")
    with pytest.raises(ValueError):
        CG.CodegenQsat(c, "E" * 12 + "AEAE")

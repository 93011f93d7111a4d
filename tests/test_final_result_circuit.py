"""QSAT results pinned by the reference's
test_opencl_quant_reducer_final_result_with_circuit (qsat.rs:6033-6267).

All twelve vectors run here.  The reference test hands its reducer an
already-decided prefix (the first `solution_bits` inputs, with its
FinalResult) and checks final_result_with_circuit (qsat.rs:1266-1320): when
the first quantifier block continues below the prefix and the prefix has a
solution, the reducer evaluates the circuit over the remaining inputs and
joins the tail's FinalResult to the prefix's (FinalResult::join,
qsat.rs:109-133); otherwise it passes the prefix's result through.  Here the
tail is the sub-formula below a fixed prefix, solved through
nsat_qsat_opts.prefix_bits/prefix on the GPU and by the oracle on the CPU,
then joined the same way.  Five vectors (5, 8, 9, 10, 11) are pass-through:
the first block ends with the prefix, or the prefix carries no solution, so
no circuit is evaluated and the expected result is the prefix's own.

Its circuits are specified by gen_circuit (qsat.rs:6010-6030): with sb
"solution bits" and 5 table bits,
    f(x) = T[x_sb .. x_sb+4] AND (x_0 .. x_sb-1 == solution),
    T[b] = bit rev5(b) of `values`,
built by gategen (not in this container), so the function is rebuilt here
as a gate list (AND/NOR with folded negations).  The reference's test hands
the reducer an already-decided prefix; for the cases whose first quantifier
block is existential and reaches into the table bits, and whose expected
answer has a solution, that is the same as solving the whole formula (f is
false for every other prefix), so the full QSAT answer must equal the
reference's expected FinalResult.  Those five vectors pin the enumeration
order, the quantifier tree over the table bits and the witness bit order.
"""
import json
import os

import pytest

from naivesat_b200.workloads import AND, NOR, XOR, RawBuilder
from oracle import oracle as O

HERE = os.path.dirname(os.path.abspath(__file__))


def lookup_circuit(sb, solution, values):
    """gen_circuit's function over sb + 5 inputs (input k = variable k)."""
    n = sb + 5
    rb = RawBuilder(n)
    eq = None
    for j in range(sb):
        neg = 0 if (solution >> j) & 1 else 1
        eq = rb.gate(AND, j, j, neg, neg) if eq is None else rb.gate(AND, eq, j, 0, neg)

    def rev5(b):
        return int("{:05b}".format(b)[::-1], 2)

    table, table_neg = None, 0          # OR of minterms, kept possibly complemented
    for b in range(32):
        if not (values >> rev5(b)) & 1:
            continue
        m = None
        for k in range(5):
            neg = 0 if (b >> k) & 1 else 1
            m = rb.gate(AND, sb + k, sb + k, neg, neg) if m is None else rb.gate(AND, m, sb + k, 0, neg)
        if table is None:
            table, table_neg = m, 0
        else:
            table, table_neg = rb.gate(NOR, table, m, table_neg, 0), 1     # or = not nor
    if table is None:
        rb.output(rb.gate(XOR, 0, 0))
    else:
        rb.output(rb.gate(AND, eq, table, 0, table_neg))
    return rb.fold()


def full_solve_cases():
    cases = json.load(open(os.path.join(HERE, "golden", "final_result_circuit.json")))["cases"]
    out = []
    for i, c in enumerate(cases):
        sb, q = c["circuit_solution_bits"], c["quants"]
        first = len(q) - len(q.lstrip(q[0]))
        if q[0] == "E" and len(q) == sb + 5 and first > sb and c["expected"]["solution"] is not None:
            out.append((i, c))
    return out


def test_full_solve_cases_are_present():
    assert [i for i, _ in full_solve_cases()] == [0, 1, 2, 3, 4]


def test_lookup_circuit_is_gen_circuit_function():
    _, c = full_solve_cases()[0]
    sb = c["circuit_solution_bits"]
    circ = lookup_circuit(sb, c["solution"], c["values"])
    oc = O.Circuit(circ.n, circ.gates, circ.outputs)
    for b in range(32):
        for prefix in (c["solution"], c["solution"] ^ 1, 0):
            x = prefix | (b << sb)
            t = (c["values"] >> int("{:05b}".format(b)[::-1], 2)) & 1
            assert O.eval_scalar(oc, [(x >> i) & 1 for i in range(sb + 5)])[0] == (t if prefix == c["solution"] else 0)


def test_oracle_reproduces_reference_result():
    """The oracle's QSAT on case 0 (2^33 items, about 15 s on 8 cores)."""
    _, c = full_solve_cases()[0]
    circ = lookup_circuit(c["circuit_solution_bits"], c["solution"], c["values"])
    r = O.qsat(O.Circuit(circ.n, circ.gates, circ.outputs), c["quants"], mode=1)
    assert {k: r[k] for k in ("reversed", "solution_bits", "solution")} == c["expected"]


@pytest.mark.gpu
def test_gpu_reproduces_reference_results(ctx):
    for i, c in full_solve_cases():
        circ = lookup_circuit(c["circuit_solution_bits"], c["solution"], c["values"])
        r = ctx.circuit(circ).qsat(c["quants"])
        assert {k: r[k] for k in ("reversed", "solution_bits", "solution")} == c["expected"], i


def first_block_len(q):
    return len(q) - len(q.lstrip(q[0]))


def join(a, b):
    """FinalResult::join (qsat.rs:109-133)."""
    assert a["reversed"] == b["reversed"]
    bits = a["solution_bits"] + b["solution_bits"]
    if a["solution"] is None:
        assert b["solution"] is None
        return {"reversed": a["reversed"], "solution_bits": bits, "solution": None}
    assert b["solution"] is not None
    return {"reversed": a["reversed"], "solution_bits": bits,
            "solution": (a["solution"] | (b["solution"] << a["solution_bits"])) & ((1 << bits) - 1)}


def prefix_value(solution, sb):
    """nsat's prefix (input 0 most significant) of a FinalResult solution
    (bit k = input k)."""
    return int(format(solution, "0%db" % sb)[::-1], 2)


def with_prefix(c, solve_sub):
    """The reducer's final_result_with_circuit restated over a sub-formula
    solver: returns (expected-comparable result, evaluated a circuit?)."""
    sb, q = c["circuit_solution_bits"], c["quants"]
    head = {"reversed": q[0] == "A", "solution_bits": sb,
            "solution": c["solution"] if c["expected"]["solution"] is not None else None}
    if first_block_len(q) <= sb or head["solution"] is None:
        return head, False
    sub = solve_sub(sb, prefix_value(c["solution"], sb))
    tail = {k: sub[k] for k in ("reversed", "solution_bits", "solution")}
    return join(head, tail), True


def all_cases():
    return json.load(open(os.path.join(HERE, "golden", "final_result_circuit.json")))["cases"]


def test_every_vector_through_prefix_subproblems_on_the_oracle():
    from test_shard import fix_prefix
    evaluated = []
    for i, c in enumerate(all_cases()):
        circ = lookup_circuit(c["circuit_solution_bits"], c["solution"], c["values"])

        def solve_sub(s, p):
            return O.qsat(fix_prefix(circ, s, p), c["quants"][s:], mode=1)
        got, ev = with_prefix(c, solve_sub)
        assert got == c["expected"], (i, got, c["expected"])
        if ev:
            evaluated.append(i)
    assert evaluated == [0, 1, 2, 3, 4, 6, 7]


@pytest.mark.gpu
def test_every_vector_through_prefix_subproblems_on_gpu(ctx):
    evaluated = []
    for i, c in enumerate(all_cases()):
        circ = lookup_circuit(c["circuit_solution_bits"], c["solution"], c["values"])
        h = ctx.circuit(circ)
        got, ev = with_prefix(c, lambda s, p: h.qsat(c["quants"], prefix_bits=s, prefix=p))
        assert got == c["expected"], (i, got, c["expected"])
        if ev:
            evaluated.append(i)
    assert evaluated == [0, 1, 2, 3, 4, 6, 7]

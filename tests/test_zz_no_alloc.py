"""nsat_qsat_solve_noalloc: the QSAT solve for callers that cannot call
cudaMalloc (a serving process whose device memory belongs to another
allocator or a fixed budget, where cudaMalloc/cudaFree would synchronize the
device or overrun the budget mid-request).  Its scratch is the library's
static device array, so its answers must equal the allocating
nsat_qsat_solve's, bit for bit, call after call (the array keeps the previous
call's bytes), and the oracle's where the oracle finishes in seconds.  This file is collected last on purpose."""
import pytest

from naivesat_b200 import api
from naivesat_b200 import workloads as W
from oracle import oracle as O

pytestmark = pytest.mark.gpu

KEYS = ("reversed", "solution_bits", "solution", "value")
ORACLE_KEYS = ("reversed", "solution_bits", "solution")


def cases():
    # two-level first block over 24 inputs: the tree runs through every stage,
    # the CTA level included (last-CTA tail in the static scratch)
    c24 = W.random_dag(501, 24, 600, output="live")
    yield c24, "EA" + "E" * 22, 0
    yield c24, "A" + "E" * 23, 15          # 2^9 launches joined on the host
    yield c24, W.alternating_quants(502, 24, 5), 0
    adder = W.config("c2b")                # 32 inputs, known counterexample a = 0
    yield adder, adder.quants, 0
    yield adder, "E" * 16 + "A" * 16, 0


def oracle_answer(circ, quants):
    """The oracle's FinalResult where it finishes in seconds (24 inputs), the
    adder's known counterexample (a = 0, 16 bits, reversed) otherwise."""
    if circ.n <= 24:
        return O.qsat(O.Circuit(circ.n, circ.gates, circ.outputs), quants, mode=1)
    if quants == circ.quants:
        return {"reversed": True, "solution_bits": 16, "solution": 0}
    return None


def test_noalloc_matches_allocating_solve_twice():
    with api.Context(0) as ctx:
        for circ, quants, chunk in cases():
            h = ctx.circuit(circ)
            ref = h.qsat(quants, chunk_bits=chunk)
            exp = oracle_answer(circ, quants)
            for call in range(2):
                got = h.qsat_noalloc(quants, chunk_bits=chunk)
                assert {k: got[k] for k in KEYS} == {k: ref[k] for k in KEYS}, (circ.name, quants, call)
                if exp is not None:
                    assert {k: got[k] for k in ORACLE_KEYS} == exp, (circ.name, quants, call)


def test_noalloc_boundary_launch_of_2_15_ctas():
    # one-warp CTAs over 2^35 assignments per launch: 2^15 CTAs, whose tail
    # needs 2 << 15 bytes, exactly the fixed area
    with api.Context(0, block_threads=32) as ctx:
        h = ctx.circuit(W.config("c1"))
        ref = h.qsat("E" * 36, chunk_bits=35)
        for call in range(2):
            got = h.qsat_noalloc("E" * 36, chunk_bits=35)
            assert {k: got[k] for k in KEYS} == {k: ref[k] for k in KEYS}, call


def test_noalloc_rejects_launches_beyond_the_fixed_area():
    # one-warp CTAs over 2^36 assignments per launch need 2^16 CTAs:
    # 2 << 16 = 128 KiB of scratch > 64 KiB
    with api.Context(0, block_threads=32) as ctx:
        h = ctx.circuit(W.config("c1"))
        with pytest.raises(api.NsatError, match="EUNSUPPORTED"):
            h.qsat_noalloc("E" * 36, chunk_bits=36)

"""The in-memory kernel cache is bounded (NSAT_JIT_MODULES): modules it drops
are unloaded once no circuit handle holds them.  With room for two modules,
solves that keep loading, evicting and reloading kernels still match the
oracle, and a handle keeps a module the cache dropped long ago usable."""
import os
import subprocess
import sys

import pytest

pytestmark = pytest.mark.gpu

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = r"""
import sys
sys.path.insert(0, %(root)r)
from naivesat_b200 import api, workloads as W
from oracle import oracle as O

def strip(r):
    return (r["reversed"], r["solution_bits"], r["solution"])

circs = [W.random_dag(500 + k, 18, 150 + 40 * k, output="live") for k in range(4)]
quants = ["A" + "E" * 17, "E" * 3 + "A" * 15, "AE" * 9, "E" * 18]
stop = W.lfsr_stop(4, 14, 120)
with api.Context(0) as ctx:
    held = ctx.circuit(circs[0])
    first = held.sat()
    ocs = [O.Circuit(c.n, c.gates, c.outputs) for c in circs]
    exp_sat = [O.sat_range(oc) for oc in ocs]
    exp_q = [O.qsat(oc, q, mode=1) for oc, q in zip(ocs, quants)]
    oc_stop = O.Circuit(stop.n, stop.gates, stop.outputs)
    exp_stop = O.stop_solve(stop.n, 6, O.stop_table(oc_stop), mode=1)
    for rep in range(3):
        for k, c in enumerate(circs):
            h = ctx.circuit(c)
            r = h.sat()
            assert (r["count"], r["witness"]) == exp_sat[k], (rep, k)
            r = h.qsat(quants[k])
            got = (r["reversed"], r["solution_bits"], r["solution"])
            want = (exp_q[k]["reversed"], exp_q[k]["solution_bits"], exp_q[k]["solution"])
            assert got == want, (rep, k)
            h.close()
        t = ctx.circuit(stop).stop_table(want_steps=True)
        g = t.solve(6, mode=1)
        t.close()
        assert g["found"] == (exp_stop is not None)
        if exp_stop is not None:
            assert (g["start"], g["end"], g["steps"]) == (exp_stop["start"], exp_stop["end"], exp_stop["steps"])
        r = held.sat()
        assert (r["count"], r["witness"]) == (first["count"], first["witness"]) == exp_sat[0], rep
print("ok")
"""


def test_bounded_kernel_cache_reloads_and_keeps_held_modules(tmp_path):
    env = dict(os.environ, NSAT_JIT_MODULES="2", NSAT_JIT_CACHE=str(tmp_path / "kernels"))
    r = subprocess.run([sys.executable, "-c", SCRIPT % {"root": ROOT}], env=env, capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stdout[-2000:] + r.stderr[-4000:]

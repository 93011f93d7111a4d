"""Multi-GPU sharding logic (naivesat_b200/shard.py) on CPU: the combination
of per-rank answers against the oracle, and the exchange over a real 2-rank
gloo process group."""
import json
import os
import socket

import pytest
import torch.multiprocessing as mp

from naivesat_b200 import shard
from naivesat_b200 import workloads as W
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def fix_prefix(circ, s, prefix):
    """Circuit over inputs s..n-1 of `circ` with inputs 0..s-1 fixed to the
    bits of `prefix` (input 0 most significant); constants are built from
    the first free input (NIMPL(x,x) = 0, NOR(0,0) = 1)."""
    n = circ.n
    m = n - s
    gates = [(W.NIMPL, 0, 0), (W.NOR, m, m)]          # wires m (=0) and m+1 (=1)
    wmap = {}
    for i in range(n):
        if i < s:
            wmap[i] = m + 1 if (prefix >> (s - 1 - i)) & 1 else m
        else:
            wmap[i] = i - s
    base = m + 2
    for k, (f, a, b) in enumerate(circ.gates.tolist()):
        wmap[n + k] = base + k
        gates.append((f, wmap[a], wmap[b]))
    outs = [(wmap[o], ng) for o, ng in circ.outputs.tolist()]
    return O.Circuit(m, gates, outs)


def oracle_sub(circ, quants, s, prefix):
    sub = fix_prefix(circ, s, prefix)
    return O.qsat(sub, quants[s:], mode=1)


def test_python_quant_reducer_matches_golden():
    with open(os.path.join(GOLD, "quant_reducer.json")) as f:
        cases = json.load(f)["cases"]
    for c in cases:
        qr = shard.QuantReducer(c["quants"])
        res = None
        for k, it in enumerate(c["items"]):
            qr.push(it)
            res = qr.final_result()
            if res is not None and res["solution"] is not None:
                break
        assert res == c["result"], c


@pytest.mark.parametrize("t", range(10))
def test_combine_qsat_matches_oracle(t):
    rng = W.SplitMix64(4000 + t)
    n = 14 + rng.below(4)
    c = W.random_dag(700 + t, n, 120, output="live")
    q = W.alternating_quants(800 + t, n, max_block=1 + rng.below(6))
    full = O.qsat(O.Circuit(c.n, c.gates, c.outputs), q, mode=1)
    for s in (1, 2, 3):
        subs = [oracle_sub(c, q, s, p) for p in range(1 << s)]
        got = shard.combine_qsat(q, subs)
        assert {k: got[k] for k in full} == full, (q, s, got, full)


def test_combine_sat():
    c = W.random_dag(9, 16, 100, output="live")
    oc = O.Circuit(c.n, c.gates, c.outputs)
    cnt, low = O.sat_range(oc)
    for world in (2, 4, 8):
        parts = []
        for r in range(world):
            b, e = shard.shard_range(1 << 16, world, r)
            k, w = O.sat_range(oc, b, e)
            parts.append({"count": k, "witness": w})
        got = shard.combine_sat(parts)
        assert (got["count"], got["witness"]) == (cnt, low)


def _rank_main(rank, world, port, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        c = W.random_dag(31, 18, 200, output="live")
        oc = O.Circuit(c.n, c.gates, c.outputs)
        sat = shard.sharded_sat(lambda b, e: dict(zip(("count", "witness"), O.sat_range(oc, b, e, 2))),
                                c.n, world, rank)
        q = W.alternating_quants(31, 18, 4)
        qs = shard.sharded_qsat(lambda s, p: oracle_sub(c, q, s, p), q, world, rank)
        with open(os.path.join(outdir, "rank%d.json" % rank), "w") as f:
            json.dump({"sat": sat, "qsat": qs}, f)
    finally:
        dist.destroy_process_group()


def free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def test_two_rank_gloo_exchange(tmp_path):
    world = 2
    mp.start_processes(_rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    c = W.random_dag(31, 18, 200, output="live")
    oc = O.Circuit(c.n, c.gates, c.outputs)
    cnt, low = O.sat_range(oc)
    q = W.alternating_quants(31, 18, 4)
    full = O.qsat(oc, q, mode=1)
    for r in range(world):
        with open(tmp_path / ("rank%d.json" % r)) as f:
            got = json.load(f)
        assert (got["sat"]["count"], got["sat"]["witness"]) == (cnt, low)
        assert {k: got["qsat"][k] for k in full} == full


def _find_rank_main(rank, world, port, outdir):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        out = {}
        for name, c in find_cases():
            oc = O.Circuit(c.n, c.gates, c.outputs)

            def solve(b, e):
                k, w = O.sat_range(oc, b, e, 2)
                return {"count": k, "witness": w}
            out[name] = shard.sharded_sat_find(solve, c.n, world, rank, 12)
        with open(os.path.join(outdir, "find%d.json" % rank), "w") as f:
            json.dump(out, f)
    finally:
        dist.destroy_process_group()


def find_cases():
    return [("early", W.Circuit(18, [(W.AND, 0, 2)], [(18, 0)], name="x0 and x2")),
            ("random", W.random_dag(33, 18, 300, output="live")),
            ("unsat", W.Circuit(18, [(W.NIMPL, 3, 3)], [(18, 0)], name="contradiction"))]


def test_two_rank_find_mode_stops_every_rank(tmp_path):
    """Find mode over 2 gloo ranks: with the lowest witness in rank 0's first
    chunk both ranks stop after one round (rank 1 scans one chunk, not its
    half of the space); answers equal the oracle's lowest witness; with no
    solution every chunk is scanned once."""
    world = 2
    mp.start_processes(_find_rank_main, args=(world, free_port(), str(tmp_path)), nprocs=world,
                       join=True, start_method="spawn")
    got = []
    for r in range(world):
        with open(tmp_path / ("find%d.json" % r)) as f:
            got.append(json.load(f))
    for name, c in find_cases():
        cnt, low = O.sat_range(O.Circuit(c.n, c.gates, c.outputs))
        for r in range(world):
            assert (got[r][name]["satisfiable"], got[r][name]["witness"]) == (low is not None, low), (name, r)
        if name == "early":
            assert low == 5
            assert all(got[r][name]["rounds"] == 1 and got[r][name]["scanned"] == 1 << 12 for r in range(world))
        if name == "unsat":
            assert sum(got[r][name]["scanned"] for r in range(world)) == 1 << 18

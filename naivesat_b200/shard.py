"""Multi-GPU sharding of the SAT and QSAT searches: one process per GPU,
no data-path collective, one small exchange of per-rank answers.

- SAT, count mode: rank r scans the contiguous index range
  [r*2^n/W, (r+1)*2^n/W); the ranks' (count, lowest witness) are combined
  by sum and min.
- SAT, find mode: chunks are dealt round-robin and the ranks exchange their
  lowest witness after every round, so all of them stop once any has one.
- QSAT: rank r fixes the outermost log2(W) inputs to r (input 0 most
  significant) and solves the sub-formula below them
  (nsat_qsat_opts.prefix_bits/prefix); the W sub-answers, in rank order, are
  combined by a forall/exists reducer over those outer inputs, joining the
  witness bits of the deciding rank when the first quantifier block reaches
  below the split (the arrangement of MainCPUQuantReducer, qsat.rs:1327-1397).

The per-rank solvers are callables, so the combination logic runs the same
with the CUDA solver or, in tests, with any other implementation.  The
exchange uses torch.distributed (NCCL across GPUs, gloo on CPU).
"""


class QuantReducer:
    """Streaming forall/exists reducer over items pushed in index order
    (the semantics of QuantReducer, qsat.rs:172-291)."""

    def __init__(self, quants):
        q = [1 if ch in "Aa" else 0 for ch in quants] if isinstance(quants, str) else [int(x) for x in quants]
        self.nq = len(q)
        fb = 0
        while fb < self.nq and q[fb] == q[0]:
            fb += 1
        self.first_bits = fb
        self.q = q[::-1]
        self.r = list(self.q)
        self.all_mask = (1 << self.nq) - 1
        self.first_mask = ((1 << fb) - 1) << (self.nq - fb)
        self.other_mask = self.all_mask & ~self.first_mask
        self.start = 0
        self.started = False
        self.solution = None

    def is_end(self):
        return self.started and (self.start & self.all_mask) == 0

    def push(self, item):
        assert not self.is_end()
        self.started = True
        index, prev = self.start, 1 if item else 0
        for i in range(self.nq):
            q, r = self.q[i], self.r[i]
            prev = (r & prev) | ((r ^ prev) & (1 - q))
            self.r[i] = prev
            if index & 1 == 0:
                break
            index >>= 1
            self.r[i] = q
        if self.solution is None and (self.start & self.other_mask) == self.other_mask and (prev ^ self.q[-1]):
            v = self.start >> (self.nq - self.first_bits)
            self.solution = int(format(v, "0%db" % self.first_bits)[::-1], 2) if self.first_bits else 0
        self.start += 1

    def final_result(self):
        if not (self.is_end() or self.solution is not None):
            return None
        return {"reversed": bool(self.q[-1]), "solution_bits": self.first_bits, "solution": self.solution}


def shard_range(total, world, rank):
    """Contiguous, equal, power-of-two aligned slice of [0, total)."""
    assert world & (world - 1) == 0 and total % world == 0
    per = total // world
    return rank * per, (rank + 1) * per


def combine_sat(results):
    """results: per rank, in rank order, dicts with count and witness."""
    count = sum(r["count"] for r in results)
    lows = [r["witness"] for r in results if r["witness"] is not None]
    return {"count": count, "witness": min(lows) if lows else None, "satisfiable": bool(lows)}


def first_block(quants):
    q = quants.upper()
    f = 0
    while f < len(q) and q[f] == q[0]:
        f += 1
    return f


def combine_qsat(quants, sub_results):
    """Combine the sub-formula answers of ranks 0..W-1 (rank r fixed the
    outermost log2(W) inputs to r).  Each sub-result carries `reversed`,
    `solution_bits`, `solution` of the formula below the prefix."""
    world = len(sub_results)
    s = world.bit_length() - 1
    assert 1 << s == world and s >= 1
    quants = quants.upper()
    f = first_block(quants)
    qr = QuantReducer(quants[:s])
    for r, sub in enumerate(sub_results):
        value = (sub["solution"] is not None) ^ sub["reversed"]
        qr.push(value)
        fr = qr.final_result()
        if fr is None:
            continue
        sol = fr["solution"]
        if sol is not None and f > s:
            # the first block continues below the split: the deciding rank's
            # sub-formula starts with the rest of it
            sol |= sub["solution"] << s
            sol &= (1 << f) - 1
        return {"reversed": quants[0] == "A", "solution_bits": f, "solution": sol,
                "value": (sol is not None) ^ (quants[0] == "A")}
    raise AssertionError("reducer did not finish")


def exchange(obj, world):
    """All-gather of a small picklable object over the default process group."""
    if world == 1:
        return [obj]
    import torch.distributed as dist
    out = [None] * world
    dist.all_gather_object(out, obj)
    return out


def sharded_sat(solve_range, n, world, rank):
    """solve_range(begin, end) -> {count, witness}; returns the whole answer
    on every rank."""
    begin, end = shard_range(1 << n, world, rank)
    mine = solve_range(begin, end)
    return combine_sat(exchange({"count": mine["count"], "witness": mine["witness"]}, world))


def sharded_sat_find(solve_range, n, world, rank, chunk_bits):
    """Find mode (the lowest witness) with a stop shared by every rank, the
    arrangement of the reference's ParSeq mapper, which hands args to the
    free device and stops all of them once one has a witness (main.rs:205-264).
    The index space is cut into chunks of 2^chunk_bits; in round t rank r
    scans chunk t*world + r, so the ranks move through the space together;
    after each round the ranks exchange their lowest witness, and they all
    stop once one exists: every chunk below it was scanned in that round or
    earlier.  solve_range(begin, end) -> {witness, count} (find mode: the
    count covers what the solver scanned).  Returns the answer on every rank
    with this rank's share of the work (scanned assignments, rounds)."""
    cb = min(chunk_bits, n)
    nchunks = 1 << (n - cb)
    mine, count, scanned, t = None, 0, 0, 0
    while True:
        c = t * world + rank
        if c < nchunks and mine is None:
            r = solve_range(c << cb, (c + 1) << cb)
            count += r["count"]
            scanned += 1 << cb
            mine = r["witness"]
        t += 1
        lows = [w for w in exchange(mine, world) if w is not None]
        if lows or t * world >= nchunks:
            return {"satisfiable": bool(lows), "witness": min(lows) if lows else None,
                    "scanned": scanned, "rounds": t, "count_scanned": count}


def sharded_qsat(solve_prefix, quants, world, rank):
    """solve_prefix(prefix_bits, prefix) -> sub-formula answer; returns the
    whole answer on every rank (world a power of two, >= 2)."""
    if world == 1:
        r = solve_prefix(0, 0)
        return {k: r[k] for k in ("reversed", "solution_bits", "solution", "value")}
    s = world.bit_length() - 1
    mine = solve_prefix(s, rank)
    subs = exchange({k: mine[k] for k in ("reversed", "solution_bits", "solution")}, world)
    return combine_qsat(quants, subs)

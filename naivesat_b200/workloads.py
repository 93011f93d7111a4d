"""Seeded synthetic circuits for the benchmark configurations.

The reference measures on prime-factoring circuit files that are not
available (benchmarks.txt:3-57); these generators stand in for them with the
shapes the benchmark configurations name.  All randomness comes from
splitmix64 so the circuits are identical on every machine.

Circuits are returned in the flat encoding of include/nsat.h: gates (g,3)
[func, i0, i1] with func 0=AND 1=NOR 2=NIMPL 3=XOR, outputs (o,2) [wire, neg].
Generators first build "raw" gates whose fan-ins may be negated, then fold
those negations forward (gatesim gates have no input negation).
"""
import math

import numpy as np

AND, NOR, NIMPL, XOR = 0, 1, 2, 3
MASK64 = (1 << 64) - 1


class SplitMix64:
    def __init__(self, seed):
        self.s = seed & MASK64

    def next(self):
        self.s = (self.s + 0x9E3779B97F4A7C15) & MASK64
        z = self.s
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def below(self, k):
        """Uniform integer in [0, k) (rejection sampling, unbiased)."""
        if k <= 1:
            return 0
        lim = (1 << 64) - ((1 << 64) % k)
        while True:
            v = self.next()
            if v < lim:
                return v % k


def _gate(f, a, b):
    if f == AND:
        return a & b
    if f == NOR:
        return 1 - (a | b)
    if f == NIMPL:
        return a & (1 - b)
    return a ^ b


class Circuit:
    """Canonical (normalised) circuit: n inputs, gates, outputs, optional quantifiers."""

    def __init__(self, n, gates, outputs, quants=None, name=""):
        self.n = int(n)
        self.gates = np.ascontiguousarray(np.asarray(gates, dtype=np.uint32).reshape(-1, 3))
        self.outputs = np.ascontiguousarray(np.asarray(outputs, dtype=np.uint32).reshape(-1, 2))
        self.quants = quants
        self.name = name

    @property
    def num_gates(self):
        return int(self.gates.shape[0])

    def eval_bits(self, bits):
        """Scalar evaluation; bits[i] is input i.  Returns the output bits."""
        w = list(bits) + [0] * self.num_gates
        n = self.n
        for k, (f, a, b) in enumerate(self.gates.tolist()):
            w[n + k] = _gate(f, w[a], w[b])
        return [w[o] ^ (ng & 1) for o, ng in self.outputs.tolist()]


class RawBuilder:
    """Gates with optionally negated fan-ins; `fold()` makes a canonical Circuit."""

    def __init__(self, n):
        self.n = n
        self.raw = []        # (func, a, na, b, nb)
        self.outs = []       # (wire, neg)

    def gate(self, f, a, b, na=0, nb=0):
        self.raw.append((f, a, int(na), b, int(nb)))
        return self.n + len(self.raw) - 1

    def output(self, w, neg=0):
        self.outs.append((w, int(neg)))

    def fold(self, quants=None, name=""):
        """Fold fan-in negations into the gate functions (gatesim has none):
        each wire carries an `inv` flag (stored value is the complement of the
        intended one); every gate is re-expressed as one of AND/NOR/NIMPL/XOR
        over its stored inputs, possibly with an output complement."""
        n = self.n
        inv = [0] * (n + len(self.raw))
        gates = []
        canon = _canonical_table()
        for k, (f, a, na, b, nb) in enumerate(self.raw):
            g, swap, oneg = canon[(f, na ^ inv[a], nb ^ inv[b])]
            gates.append((g, b, a) if swap else (g, a, b))
            inv[n + k] = oneg
        outputs = [(w, ng ^ inv[w]) for (w, ng) in self.outs]
        return Circuit(n, gates, outputs, quants=quants, name=name)


_CANON = None


def _canonical_table():
    """(func, negate i0, negate i1) -> (gatesim func, swap inputs, complement
    output) with the same truth table over the un-negated inputs."""
    global _CANON
    if _CANON is None:
        _CANON = {}
        for f in (AND, NOR, NIMPL, XOR):
            for ea in (0, 1):
                for eb in (0, 1):
                    tt = [_gate(f, x ^ ea, y ^ eb) for x in (0, 1) for y in (0, 1)]
                    found = None
                    for g in (f, AND, NOR, NIMPL, XOR):
                        for swap in (0, 1):
                            for oneg in (0, 1):
                                if all(((_gate(g, y, x) if swap else _gate(g, x, y)) ^ oneg) == tt[2 * x + y]
                                       for x in (0, 1) for y in (0, 1)):
                                    found = found or (g, swap, oneg)
                    assert found is not None
                    _CANON[(f, ea, eb)] = found
    return _CANON


def random_dag_raw(rng, n, num_gates, window=64, neg_prob_quarter=True):
    """Random DAG: gate types uniform over the four, each fan-in uniform over
    the preceding `window` nodes, each negated with probability 1/4."""
    rb = RawBuilder(n)
    for k in range(num_gates):
        node = n + k
        lo = max(0, node - window)
        f = rng.below(4)
        a = lo + rng.below(node - lo)
        na = 1 if rng.below(4) == 0 else 0
        b = lo + rng.below(node - lo)
        nb = 1 if rng.below(4) == 0 else 0
        rb.gate(f, a, b, na, nb)
    return rb


def sample_words(circ, samples=4096, seed=0x5A3B1E):
    """Bit-parallel evaluation of every wire on `samples` seeded random
    assignments (Python ints as bit vectors).  Returns the list of wire values."""
    rng = SplitMix64(seed)
    full = (1 << samples) - 1
    w = []
    for _ in range(circ.n):
        v = 0
        for k in range(samples // 64):
            v |= rng.next() << (64 * k)
        w.append(v)
    for (f, a, b) in circ.gates.tolist():
        x, y = w[a], w[b]
        w.append(x & y if f == AND else full ^ (x | y) if f == NOR else x & (full ^ y) if f == NIMPL else x ^ y)
    return w, full


def last_live_gate(circ):
    """Index of the last gate whose value is not constant over 4096 seeded
    samples.  Deep random DAGs with a 64-node window lose their entropy: in
    the 3000-gate DAGs of seeds 1 and 2 more than half of the gates are
    constant on every sample, the last gate included."""
    w, full = sample_words(circ)
    for k in range(circ.num_gates - 1, -1, -1):
        v = w[circ.n + k]
        if v != 0 and v != full:
            return k
    return circ.num_gates - 1


def random_dag(seed, n, num_gates, window=64, output="last"):
    """Random DAG generator.  output="last": the single output is the last
    gate (config 0 as specified); output="live": the last gate that is not
    constant on the seeded sample (used where the last gate is constant).
    Runs the library's generator (nsat_gen_random_dag), which is bit-identical
    to random_dag_py below."""
    from . import api
    gates, outputs = api.gen_random_dag(seed, n, num_gates, window, output == "live")
    c = Circuit(n, gates, outputs, name="dag_s%d_n%d_g%d" % (seed, n, num_gates))
    c.out_gate = int(outputs[0][0]) - n
    return c


def random_dag_py(seed, n, num_gates, window=64, output="last"):
    """Pure-Python statement of random_dag (the reference for the library's
    generator)."""
    rng = SplitMix64(seed)
    rb = random_dag_raw(rng, n, num_gates, window)
    out = n + num_gates - 1
    if output == "live":
        rb.output(out)
        probe = rb.fold()
        rb.outs.clear()
        out = n + last_live_gate(probe)
    rb.output(out)
    c = rb.fold(name="dag_s%d_n%d_g%d" % (seed, n, num_gates))
    c.out_gate = out - n
    return c


def planted_dag(seed, n, num_gates, plant_bits=18, window=64):
    """Config 1: random DAG ANDed with x[0..plant_bits) == K, where K is taken
    from a seeded assignment that satisfies the DAG (so solutions exist).  The
    DAG output is its last non-constant gate (see last_live_gate)."""
    rng = SplitMix64(seed)
    rb = random_dag_raw(rng, n, num_gates, window)
    rb.output(n + num_gates - 1)
    probe = rb.fold()
    rb.outs.clear()
    dag_out = n + last_live_gate(probe)
    rb.output(dag_out)
    base = rb.fold()
    rb.outs.clear()
    tries = 0
    while True:
        x = rng.next() & ((1 << n) - 1)
        tries += 1
        bits = [(x >> i) & 1 for i in range(n)]
        w = list(bits) + [0] * base.num_gates
        for k, (f, a, b) in enumerate(base.gates.tolist()):
            w[n + k] = _gate(f, w[a], w[b])
        o, ng = base.outputs[0].tolist()
        if w[o] ^ ng:
            break
        assert tries < 10000
    K = x & ((1 << plant_bits) - 1)
    acc = dag_out
    for i in range(plant_bits):
        acc = rb.gate(AND, acc, i, 0, 0 if (K >> i) & 1 else 1)
    rb.output(acc)
    c = rb.fold(name="planted_s%d_n%d_g%d" % (seed, n, num_gates))
    c.plant_k = K
    c.plant_x = x
    return c


def adder_qsat(force_b15_zero=False, target=0xBEEF):
    """Config 2a/2b: forall a[0..16) exists b[16..32): (a+b) mod 2^16 == target,
    ripple-carry adder (LSB = lowest input) plus an XNOR/AND comparator.
    With force_b15_zero the adder sees b15 = 0 (input 31 stays unused)."""
    n = 32
    rb = RawBuilder(n)
    a = list(range(16))
    b = list(range(16, 32))
    s = []
    carry = None   # (wire, neg)
    for i in range(16):
        if force_b15_zero and i == 15:
            if carry is None:
                s.append((a[i], 0))
            else:
                s.append((rb.gate(XOR, a[i], carry[0], 0, carry[1]), 0))
            continue
        t = rb.gate(XOR, a[i], b[i])
        if carry is None:
            s.append((t, 0))
            carry = (rb.gate(AND, a[i], b[i]), 0)
        else:
            s.append((rb.gate(XOR, t, carry[0], 0, carry[1]), 0))
            g = rb.gate(AND, a[i], b[i])
            p = rb.gate(AND, t, carry[0], 0, carry[1])
            carry = (rb.gate(NOR, g, p), 1)       # OR = NOR with the complement
    # comparator: AND over literals (s_i or not s_i)
    lits = [(w, ng ^ (0 if (target >> i) & 1 else 1)) for i, (w, ng) in enumerate(s)]
    acc = rb.gate(AND, lits[0][0], lits[1][0], lits[0][1], lits[1][1])
    for (w, ng) in lits[2:]:
        acc = rb.gate(AND, acc, w, 0, ng)
    rb.output(acc)
    quants = "A" * 16 + "E" * 16
    return rb.fold(quants=quants, name="adder_b15zero" if force_b15_zero else "adder")


def alternating_quants(seed, n, max_block=6):
    rng = SplitMix64(seed ^ 0x5157A7)
    q = "A" if rng.below(2) else "E"
    out = ""
    while len(out) < n:
        ln = 1 + rng.below(max_block)
        out += q * ln
        q = "E" if q == "A" else "A"
    return out[:n]


def qsat_dag(seed, n, num_gates):
    """Config 2c: random DAG under a seeded alternating quantifier string."""
    c = random_dag(seed, n, num_gates, output="live")
    c.quants = alternating_quants(seed, n)
    c.name = "qdag_s%d_n%d_g%d" % (seed, n, num_gates)
    return c


def _eq_chain(rb, n, pattern):
    """AND over the literals s_i == pattern_i of the state inputs."""
    acc = rb.gate(AND, 0, 1, 0 if pattern & 1 else 1, 0 if (pattern >> 1) & 1 else 1)
    for i in range(2, n):
        acc = rb.gate(AND, acc, i, 0, 0 if (pattern >> i) & 1 else 1)
    return acc


def lfsr_stop(seed, n=24, mixer_gates=300):
    """Config 3a: next = Fibonacci LFSR(s) XOR mixer(s), STOP = (s == P).
    Runs the library's generator (nsat_gen_lfsr_stop), bit-identical to
    lfsr_stop_py below."""
    from . import api
    gates, outputs, pattern = api.gen_lfsr_stop(seed, n, mixer_gates)
    c = Circuit(n, gates, outputs, name="lfsr_s%d_n%d" % (seed, n))
    c.pattern = pattern
    return c


def lfsr_stop_py(seed, n=24, mixer_gates=300):
    """Pure-Python statement of lfsr_stop."""
    rng = SplitMix64(seed)
    taps = {n - 1}
    while len(taps) < 4:
        taps.add(rng.below(n - 1))
    taps = sorted(taps)
    pattern = rng.next() & ((1 << n) - 1)
    rb = random_dag_raw(rng, n, mixer_gates)
    mix_first = n + (mixer_gates - n)    # wire of the first of the last n mixer gates
    fb = rb.gate(XOR, taps[0], taps[1])
    for t in taps[2:]:
        fb = rb.gate(XOR, fb, t)
    nxt = []
    for i in range(n):
        lf = fb if i == 0 else (i - 1)
        nxt.append(rb.gate(XOR, lf, mix_first + i))
    stop = _eq_chain(rb, n, pattern)
    for w in nxt:
        rb.output(w)
    rb.output(stop)
    c = rb.fold(name="lfsr_s%d_n%d" % (seed, n))
    c.pattern = pattern
    c.taps = taps
    return c


def counter_stop(n=24):
    """Config 3b: next = s + 1 mod 2^n, STOP = (s == 2^n - 1)."""
    rb = RawBuilder(n)
    nxt = [(0, 1)]            # bit 0 = not s0 (an output complement)
    carry = (0, 0)            # carry into bit 1 = s0
    for i in range(1, n):
        nxt.append((rb.gate(XOR, i, carry[0], 0, carry[1]), 0))
        if i < n - 1:
            carry = (rb.gate(AND, i, carry[0], 0, carry[1]), 0)
    stop = _eq_chain(rb, n, (1 << n) - 1)
    for (w, ng) in nxt:
        rb.output(w, ng)
    rb.output(stop)
    return rb.fold(name="counter_n%d" % n)


def identity_stop(n, stop_input=0):
    """Outputs 0..n-1 copy the inputs, output n copies input `stop_input`:
    table entry s is s | (bit stop_input of s) << n (enumeration layout pin)."""
    return Circuit(n, np.zeros((0, 3), dtype=np.uint32),
                   [(i, 0) for i in range(n)] + [(stop_input, 0)], name="identity%d" % n)


def config(name):
    """The benchmark configurations by name."""
    if name == "c0":
        return random_dag(0, 24, 500)
    if name == "c1":
        return planted_dag(1, 36, 3000)
    if name == "c1_twin":
        return random_dag(2, 36, 3000, output="live")
    if name == "c2a":
        return adder_qsat(False)
    if name == "c2b":
        return adder_qsat(True)
    if name == "c2c":
        return qsat_dag(3, 30, 1500)
    if name == "c3a":
        return lfsr_stop(4, 24, 300)
    if name == "c3b":
        return counter_stop(24)
    raise KeyError(name)


def serving_requests(count, seed=2024, rate_hz=100.0, n_range=(18, 34), g_range=(100, 4000),
                     mix=(0.7, 0.2, 0.1), stop_n_range=(12, 20)):
    """Config 4: `count` requests with Poisson arrivals at `rate_hz`: SAT /
    QSAT / SATOSTOP in proportions `mix`; SAT and QSAT circuits have
    n ~ U[n_range] inputs and G ~ log-uniform[g_range] gates (the config-0
    generator, per-request seeds, live output), QSAT quantifiers are seeded
    random; SATOSTOP circuits are LFSR+mixer next-state circuits with
    n ~ U[stop_n_range] state bits and the top n/2 bits unknown."""
    rng = SplitMix64(seed)
    reqs = []
    t = 0.0
    for i in range(count):
        # exponential inter-arrival time from a uniform in (0, 1]
        u = (rng.next() >> 11) / float(1 << 53)
        t += -math.log(1.0 - u) / rate_hz if u < 1.0 else 0.0
        r = (rng.next() >> 11) / float(1 << 53)
        kind = "sat" if r < mix[0] else "qsat" if r < mix[0] + mix[1] else "stop"
        rseed = rng.next() & 0xFFFFFFFF
        if kind == "stop":
            n = stop_n_range[0] + rng.below(stop_n_range[1] - stop_n_range[0] + 1)
            g = int(math.exp(math.log(50) + (rng.next() >> 11) / float(1 << 53) * (math.log(1000) - math.log(50))))
            c = lfsr_stop(rseed, n, max(g, n + 1))
            reqs.append({"arrival_s": t, "kind": "stop", "circ": c, "quants": None, "unknowns": n // 2,
                         "seed": rseed})
            continue
        n = n_range[0] + rng.below(n_range[1] - n_range[0] + 1)
        lg = math.log(g_range[0]) + (rng.next() >> 11) / float(1 << 53) * (math.log(g_range[1]) - math.log(g_range[0]))
        g = int(math.exp(lg))
        c = random_dag(rseed, n, g, output="live")
        quants = None
        if kind == "qsat":
            qr = SplitMix64(rseed ^ 0xA5A5)
            quants = "".join("A" if qr.below(2) else "E" for _ in range(n))
            c.quants = quants
        reqs.append({"arrival_s": t, "kind": kind, "circ": c, "quants": quants, "unknowns": 0, "seed": rseed})
    return reqs

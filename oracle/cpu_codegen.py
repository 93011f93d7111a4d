"""Generated-code CPU baseline for exhaustive SAT and QSAT.

TEST INFRASTRUCTURE ONLY: a timed CPU baseline beside the oracle (the
checker).  Only tests/ and bench.py's CPU-baseline and reference legs import
it; the product package never does.

It restates how the reference's CPU path evaluates a circuit.  naivesat with
`-t cpu` (main.rs:281-287, 106-155) builds the circuit with gatenative's
CPUBuilder: the builder writes C source for that one circuit, with every gate
as one bitwise operation on a machine vector word (TYPE_LEN assignments per
word).  The elem inputs (0..e) are enumerated inside one call, from lane
constants and the element index.  The arg inputs (e..n) are fixed per call.
The builder compiles that source with the host C compiler and runs the calls
in parallel across args (rayon in the reference, OpenMP here).  gatenative
0.2.0 itself is not in this container, so this module writes its own source
in that shape:

* the widest vector type of the host: AVX-512 (512 assignments per word),
  else AVX2 (256), else u64;
* straight-line code, one vector operation per live gate, in gate order
  (And a&b, Nor ~(a|b), Nimpl a&~b, Xor a^b);
* per call (arg): the inputs e..n-1 are broadcast once, and the loop over the
  call's words computes the elem inputs above the vector width from the word
  index;
* per word: popcount and the lowest set bit, summed and min-reduced per call
  (count mode and lowest witness, as the CUDA path reports them).

QSAT (naiveqsat with `-t cpu`, qsat.rs:1327-1397: MainCPUQuantReducer over
CPU-built calls) uses the same evaluation in v-order: input i is bit n-1-i of
the item index, the call's items are the last e inputs (input n-1 the lowest
bit) and its arg the first n-e (input 0 the highest bit).  Each call reduces
its items through the quantifier levels below the first quantifier block
(the unit level) with bit operations: six levels inside each 64-bit word,
the lanes of the vector, then a stack across the call's vector words.  The
calls' unit values, in order, go through the QuantReducer of the first
block, which gives the reference's FinalResult.  Units must be at least one
vector word (the first block ends 9 or more inputs above the last).

The generated file is compiled with `gcc -O3 -march=native -fopenmp` into a
temporary directory and loaded with ctypes.  Compile time is not part of any
timing, as in the reference, whose build step comes before its timer
(main.rs:122-125).
"""
import ctypes as C
import os
import shutil
import subprocess
import tempfile

LANE_PAT = [0xAAAAAAAAAAAAAAAA, 0xCCCCCCCCCCCCCCCC, 0xF0F0F0F0F0F0F0F0,
            0xFF00FF00FF00FF00, 0xFFFF0000FFFF0000, 0xFFFFFFFF00000000]

_PRELUDE = r"""
#include <stdint.h>
#include <immintrin.h>
#ifdef _OPENMP
#include <omp.h>
#endif
#if defined(__AVX512F__)
typedef __m512i V;
#define VB 9
#define NW 8
#define AND(a, b) _mm512_and_si512(a, b)
#define NOR(a, b) _mm512_xor_si512(_mm512_or_si512(a, b), _mm512_set1_epi64(-1))
#define NIMPL(a, b) _mm512_andnot_si512(b, a)
#define XOR(a, b) _mm512_xor_si512(a, b)
#define NOT(a) _mm512_xor_si512(a, _mm512_set1_epi64(-1))
#define BCAST(x) _mm512_set1_epi64((long long)(x))
#define STORE(p, v) _mm512_storeu_si512((void*)(p), v)
static inline V lane_bit(int b) {
    long long w[8];
    for (int k = 0; k < 8; k++) w[k] = ((k >> (b - 6)) & 1) ? -1LL : 0LL;
    return _mm512_loadu_si512((const void*)w);
}
#elif defined(__AVX2__)
typedef __m256i V;
#define VB 8
#define NW 4
#define AND(a, b) _mm256_and_si256(a, b)
#define NOR(a, b) _mm256_xor_si256(_mm256_or_si256(a, b), _mm256_set1_epi64x(-1))
#define NIMPL(a, b) _mm256_andnot_si256(b, a)
#define XOR(a, b) _mm256_xor_si256(a, b)
#define NOT(a) _mm256_xor_si256(a, _mm256_set1_epi64x(-1))
#define BCAST(x) _mm256_set1_epi64x((long long)(x))
#define STORE(p, v) _mm256_storeu_si256((void*)(p), v)
static inline V lane_bit(int b) {
    long long w[4];
    for (int k = 0; k < 4; k++) w[k] = ((k >> (b - 6)) & 1) ? -1LL : 0LL;
    return _mm256_loadu_si256((const void*)w);
}
#else
typedef uint64_t V;
#define VB 6
#define NW 1
#define AND(a, b) ((a) & (b))
#define NOR(a, b) (~((a) | (b)))
#define NIMPL(a, b) ((a) & ~(b))
#define XOR(a, b) ((a) ^ (b))
#define NOT(a) (~(a))
#define BCAST(x) ((uint64_t)(x))
#define STORE(p, v) (*(p) = (v))
static inline V lane_bit(int b) { return 0; }
#endif

static inline V in_bit(int b, uint64_t word) {
    static const uint64_t pat[6] = {0xAAAAAAAAAAAAAAAAull, 0xCCCCCCCCCCCCCCCCull, 0xF0F0F0F0F0F0F0F0ull,
                                    0xFF00FF00FF00FF00ull, 0xFFFF0000FFFF0000ull, 0xFFFFFFFF00000000ull};
    if (b < 6) return BCAST(pat[b]);
    if (b < VB) return lane_bit(b);
    return BCAST(((word >> (b - VB)) & 1) ? ~0ull : 0ull);
}

int nsat_cg_vector_bits(void) { return VB; }
"""


def c_source(circ, elem_bits):
    """C source of the SAT evaluator of `circ` (output 0) with elem_bits
    elem inputs per call."""
    n = circ.n
    gates = circ.gates
    out_wire, out_neg = circ.outputs[0]
    live = [False] * (n + len(gates))
    live[out_wire] = True
    for k in range(len(gates) - 1, -1, -1):
        if live[n + k]:
            _, a, b = gates[k]
            live[a] = live[b] = True
    ops = ("AND", "NOR", "NIMPL", "XOR")
    L = [_PRELUDE]
    L.append("#define EB %d\n" % elem_bits)
    L.append("static void call(uint64_t arg, uint64_t* cnt, uint64_t* low) {")
    # arg inputs: broadcast once per call
    for i in range(n):
        if live[i] and i >= elem_bits:
            L.append("    const V w%d = BCAST(((arg >> %d) & 1) ? ~0ull : 0ull);" % (i, i - elem_bits))
    L.append("    uint64_t c = 0, lo = ~0ull;")
    L.append("    for (uint64_t word = 0; word < (1ull << (EB - VB)); word++) {")
    for i in range(min(n, elem_bits)):
        if live[i]:
            L.append("        const V w%d = in_bit(%d, word);" % (i, i))
    for k, (f, a, b) in enumerate(gates):
        if live[n + k]:
            L.append("        const V w%d = %s(w%d, w%d);" % (n + k, ops[f], a, b))
    L.append("        V o = %s;" % (("NOT(w%d)" % out_wire) if out_neg else ("w%d" % out_wire)))
    L.append("        uint64_t ow[NW];")
    L.append("        STORE(ow, o);")
    L.append("        for (int k = 0; k < NW; k++) {")
    L.append("            const uint64_t x = ow[k];")
    L.append("            if (x) {")
    L.append("                c += (uint64_t)__builtin_popcountll(x);")
    L.append("                if (lo == ~0ull) lo = (word << VB) | ((uint64_t)k << 6) | (uint64_t)__builtin_ctzll(x);")
    L.append("            }")
    L.append("        }")
    L.append("    }")
    L.append("    *cnt = c;")
    L.append("    *low = lo == ~0ull ? lo : (lo | (arg << EB));")
    L.append("}")
    L.append("""
int nsat_cg_sat_args(uint64_t a0, uint64_t a1, int threads, uint64_t* count, uint64_t* lowest) {
    uint64_t gc = 0, gl = ~0ull;
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1) reduction(+ : gc) reduction(min : gl)
#endif
    for (uint64_t a = a0; a < a1; a++) {
        uint64_t c, l;
        call(a, &c, &l);
        gc += c;
        if (l < gl) gl = l;
    }
    *count = gc;
    *lowest = gl;
    return 0;
}
""")
    return "\n".join(L)


def compiler():
    return shutil.which("gcc") or shutil.which("cc")


class CodegenSat:
    """A circuit's generated SAT evaluator, compiled and loaded.  Calls
    enumerate 2^elem_bits assignments each (the reference's `-e`, clamped
    as do_command clamps it, main.rs:269-275)."""

    def __init__(self, circ, elem_bits=None, flags=("-O3", "-march=native", "-fopenmp")):
        n = circ.n
        e = 24 if elem_bits is None else elem_bits
        if e >= n:
            e = n - 1
        self.circ = circ
        self.e = e
        self.dir = tempfile.mkdtemp(prefix="nsat_cg_")
        src = os.path.join(self.dir, "cg.c")
        so = os.path.join(self.dir, "cg.so")
        with open(src, "w") as f:
            f.write(c_source(circ, e))
        cc = compiler()
        if cc is None:
            raise RuntimeError("no C compiler for the generated-code CPU baseline")
        subprocess.run([cc, *flags, "-fPIC", "-shared", "-o", so, src], check=True)
        self.lib = C.CDLL(so)
        self.lib.nsat_cg_sat_args.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.POINTER(C.c_uint64),
                                              C.POINTER(C.c_uint64)]
        self.vector_bits = 1 << self.lib.nsat_cg_vector_bits()
        if e < self.lib.nsat_cg_vector_bits():
            raise ValueError("elem bits below the vector width")

    def sat_args(self, a0, a1, threads=0):
        """Count and lowest witness over args [a0, a1), i.e. assignments
        [a0 << e, a1 << e)."""
        cnt, low = C.c_uint64(), C.c_uint64()
        self.lib.nsat_cg_sat_args(a0, a1, threads, C.byref(cnt), C.byref(low))
        return cnt.value, (None if low.value == (1 << 64) - 1 else low.value)

    def close(self):
        if self.dir:
            shutil.rmtree(self.dir, ignore_errors=True)
            self.dir = None

    def __del__(self):
        self.close()


def first_block(quants):
    """Length of the first quantifier block of a quantifier string."""
    return len(quants) - len(quants.lstrip(quants[0]))


def c_source_qsat(circ, elem_bits, quants):
    """C source of the QSAT call of `circ` (output 0) under `quants`: every
    call evaluates the 2^elem_bits items of one arg in v-order and reduces
    them through min(m, elem_bits) quantifier levels, m = n - first block,
    writing one byte per value (2^(elem_bits - levels) per call)."""
    n = circ.n
    e = elem_bits
    m = n - first_block(quants)
    L = min(m, e)
    gates = circ.gates
    out_wire, out_neg = circ.outputs[0]
    live = [False] * (n + len(gates))
    live[out_wire] = True
    for k in range(len(gates) - 1, -1, -1):
        if live[n + k]:
            _, a, b = gates[k]
            live[a] = live[b] = True
    ops = ("AND", "NOR", "NIMPL", "XOR")
    # level k (bit k of the item index) belongs to input n-1-k
    qa = [1 if quants[n - 1 - k] in "Aa" else 0 for k in range(n)]
    S = [_PRELUDE]
    S.append("#define EB %d\n#define LV %d" % (e, L))
    S.append("static const unsigned char qa[%d] = {%s};" % (n, ", ".join(str(v) for v in qa)))
    S.append("static inline uint64_t comb(int lvl, uint64_t a, uint64_t b) { return qa[lvl] ? (a & b) : (a | b); }")
    S.append("static void qcall(uint64_t arg, unsigned char* out) {")
    for i in range(n - e):
        if live[i]:
            S.append("    const V w%d = BCAST(((arg >> %d) & 1) ? ~0ull : 0ull);" % (i, n - e - 1 - i))
    S.append("    unsigned char sv[64]; int sl[64]; int sp = 0; uint64_t no = 0;")
    S.append("    for (uint64_t word = 0; word < (1ull << (EB - VB)); word++) {")
    for i in range(n - e, n):
        if live[i]:
            S.append("        const V w%d = in_bit(%d, word);" % (i, n - 1 - i))
    for k, (f, a, b) in enumerate(gates):
        if live[n + k]:
            S.append("        const V w%d = %s(w%d, w%d);" % (n + k, ops[f], a, b))
    S.append("        V o = %s;" % (("NOT(w%d)" % out_wire) if out_neg else ("w%d" % out_wire)))
    S.append("        uint64_t ow[NW];")
    S.append("        STORE(ow, o);")
    # levels 0..5 inside each 64-bit word, then the vector's lanes
    S.append("        for (int j = 0; j < NW; j++) {")
    S.append("            uint64_t x = ow[j];")
    S.append("            for (int l = 0; l < 6; l++) x = comb(l, x, x >> (1 << l));")
    S.append("            ow[j] = x & 1;")
    S.append("        }")
    S.append("        for (int l = 6; l < VB; l++) {")
    S.append("            const int st = 1 << (l - 6);")
    S.append("            for (int j = 0; j < NW; j += 2 * st) ow[j] = comb(l, ow[j], ow[j + st]);")
    S.append("        }")
    S.append("        unsigned char v = (unsigned char)ow[0];")
    S.append("        int lvl = VB;")
    S.append("        while (lvl < LV && sp > 0 && sl[sp - 1] == lvl) { v = (unsigned char)comb(lvl, sv[sp - 1], v); sp--; lvl++; }")
    S.append("        if (lvl == LV) out[no++] = v;")
    S.append("        else { sv[sp] = v; sl[sp] = lvl; sp++; }")
    S.append("    }")
    S.append("}")
    S.append("""
int nsat_cg_qsat_args(uint64_t a0, uint64_t a1, int threads, unsigned char* out) {
    const uint64_t per = 1ull << (EB - LV);
#ifdef _OPENMP
    if (threads <= 0) threads = omp_get_max_threads();
#pragma omp parallel for num_threads(threads) schedule(dynamic, 1)
#endif
    for (uint64_t a = a0; a < a1; a++) qcall(a, out + (a - a0) * per);
    return 0;
}
""")
    return "\n".join(S)


class CodegenQsat:
    """A circuit's generated QSAT calls under one quantifier string, compiled
    and loaded.  Calls enumerate 2^elem_bits items each (the last elem_bits
    inputs in v-order)."""

    def __init__(self, circ, quants, elem_bits=None, flags=("-O3", "-march=native", "-fopenmp")):
        import numpy as np   # noqa: F401  (used by solve)
        n = circ.n
        if len(quants) != n:
            raise ValueError("one quantifier per input")
        e = 24 if elem_bits is None else elem_bits
        if e >= n:
            e = n - 1
        self.circ, self.quants, self.e = circ, quants, e
        self.f = first_block(quants)
        self.m = n - self.f
        self.dir = tempfile.mkdtemp(prefix="nsat_cgq_")
        cc = compiler()
        if cc is None:
            raise RuntimeError("no C compiler for the generated-code CPU baseline")
        # the vector width of this host decides whether units fit whole words
        probe = os.path.join(self.dir, "vb.c")
        with open(probe, "w") as fh:
            fh.write(_PRELUDE)
        vb_so = os.path.join(self.dir, "vb.so")
        subprocess.run([cc, *flags, "-fPIC", "-shared", "-o", vb_so, probe], check=True)
        vb = C.CDLL(vb_so).nsat_cg_vector_bits()
        if self.m < vb or e < vb:
            self.close()
            raise ValueError("units smaller than a %d-bit vector word" % (1 << vb))
        src = os.path.join(self.dir, "cgq.c")
        so = os.path.join(self.dir, "cgq.so")
        with open(src, "w") as fh:
            fh.write(c_source_qsat(circ, e, quants))
        subprocess.run([cc, *flags, "-fPIC", "-shared", "-o", so, src], check=True)
        self.lib = C.CDLL(so)
        self.lib.nsat_cg_qsat_args.argtypes = [C.c_uint64, C.c_uint64, C.c_int, C.c_void_p]
        self.vector_bits = 1 << vb
        self.levels = min(self.m, e)

    def values(self, a0, a1, threads=0):
        """The reduced values of args [a0, a1), in item order (uint8)."""
        import numpy as np
        per = 1 << (self.e - self.levels)
        out = np.zeros((a1 - a0) * per, dtype=np.uint8)
        self.lib.nsat_cg_qsat_args(a0, a1, threads, out.ctypes.data)
        return out

    def solve(self, threads=0, batch_calls=None):
        """FinalResult of the whole formula.  Calls run in order, a batch at a
        time (all host threads on one batch); each batch's values are reduced
        up to the unit level and pushed into the first block's QuantReducer,
        and the solve stops once that reducer has its result, as the
        reference's reducer stops its calls (qsat.rs:1327-1397)."""
        import numpy as np
        from oracle import oracle as O
        n = self.circ.n
        calls = 1 << (n - self.e)
        span = 1 << max(0, self.m - self.e)          # calls per unit
        if batch_calls is None:
            batch_calls = max(span, min(calls, 4 * (threads or os.cpu_count() or 1)))
        batch_calls = max(span, batch_calls // span * span)
        qr = O.QuantReducer(self.quants[:self.f])
        unit = 0
        for a in range(0, calls, batch_calls):
            v = self.values(a, min(calls, a + batch_calls), threads)
            for lvl in range(self.levels, self.m):    # units that span calls
                pair = v.reshape(-1, 2)
                v = (pair[:, 0] & pair[:, 1]) if self.quants[n - 1 - lvl] in "Aa" else (pair[:, 0] | pair[:, 1])
            if len(v) % 32:
                for k, x in enumerate(v):
                    qr.push(unit + k, int(x))
            else:
                # item unit + k = bit k % 32 of word k / 32
                words = np.packbits(v.reshape(-1, 32)[:, ::-1], axis=1).view(">u4").astype(np.uint32).reshape(-1)
                qr.push_words(words, unit)
            unit += len(v)
            r = qr.final_result()
            if r is not None:
                return r
        return qr.final_result()

    def close(self):
        if getattr(self, "dir", None):
            shutil.rmtree(self.dir, ignore_errors=True)
            self.dir = None

    def __del__(self):
        self.close()

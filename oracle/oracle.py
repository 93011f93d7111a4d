"""ctypes front end of the CPU oracle (nsat_oracle.c).

TEST INFRASTRUCTURE ONLY: the checker that the CUDA path is compared against,
and the timed CPU baseline.  Only tests/, __graft_entry__.smoke() and the CPU
baseline leg of bench.py import this module; the product package never does.
"""
import ctypes as C
import os
import subprocess
import threading

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle.so")
_lock = threading.Lock()
_lib = None

U8P = C.POINTER(C.c_uint8)
U32P = C.POINTER(C.c_uint32)
U64P = C.POINTER(C.c_uint64)


class OrCircuit(C.Structure):
    _fields_ = [("n", C.c_uint32), ("g", C.c_uint32), ("gates", U32P),
                ("o", C.c_uint32), ("outputs", U32P)]


def build():
    """Compile liboracle.so with the Makefile beside this file."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    with _lock:
        if _lib is None:
            src = os.path.join(HERE, "nsat_oracle.c")
            if not os.path.exists(LIB_PATH) or os.path.getmtime(LIB_PATH) < os.path.getmtime(src):
                build()
            L = C.CDLL(LIB_PATH)
            L.or_eval_scalar.argtypes = [C.POINTER(OrCircuit), U8P, U8P]
            L.or_eval_words.argtypes = [C.POINTER(OrCircuit), U64P, U64P]
            L.or_sat_range.argtypes = [C.POINTER(OrCircuit), C.c_uint64, C.c_uint64, C.c_int,
                                       U64P, U64P]
            L.or_qr_new.argtypes = [U8P, C.c_int]
            L.or_qr_new.restype = C.c_void_p
            L.or_qr_free.argtypes = [C.c_void_p]
            L.or_qr_push.argtypes = [C.c_void_p, C.c_uint64, C.c_int]
            L.or_qr_push_words.argtypes = [C.c_void_p, U32P, C.c_uint64]
            L.or_qr_push_words_from.argtypes = [C.c_void_p, C.c_uint64, U32P, C.c_uint64]
            L.or_qr_final.argtypes = [C.c_void_p, C.POINTER(C.c_int), U32P, C.POINTER(C.c_int), U64P]
            L.or_qsat.argtypes = [C.POINTER(OrCircuit), U8P, C.c_int, C.c_int, C.POINTER(C.c_int),
                                  U32P, C.POINTER(C.c_int), U64P]
            L.or_stop_table.argtypes = [C.POINTER(OrCircuit), C.c_int, U64P]
            L.or_stop_solve.argtypes = [C.c_uint32, C.c_uint32, U64P, C.c_int, C.c_int,
                                        C.POINTER(C.c_int), U64P, U64P, U64P, U32P]
            L.or_stop_replay.argtypes = [C.POINTER(OrCircuit), C.c_uint64, C.c_uint64, U64P, U64P]
            L.or_memimage_get.argtypes = [U64P, C.c_uint32, C.c_uint64]
            L.or_memimage_get.restype = C.c_uint64
            L.or_memimage_set.argtypes = [U64P, C.c_uint32, C.c_uint64, C.c_uint64]
            L.or_greedy_partitioned.argtypes = [U64P, C.c_uint32, C.c_uint32, C.c_uint32,
                                                C.POINTER(C.c_uint64), C.POINTER(C.c_uint64),
                                                C.POINTER(C.c_uint32), C.POINTER(C.c_uint32)]
            L.or_memimage_find_solution.argtypes = [U64P, C.c_uint32, C.c_uint64, C.c_uint64,
                                                    C.c_uint32, U64P, U64P]
            _lib = L
    return _lib


def _ptr(a, t):
    return a.ctypes.data_as(t)


class Circuit:
    """A circuit in the shared flat encoding: gates (g,3) [func,i0,i1] and
    outputs (o,2) [wire,negated]."""

    def __init__(self, n, gates, outputs):
        self.n = int(n)
        self.gates = np.ascontiguousarray(np.asarray(gates, dtype=np.uint32).reshape(-1, 3))
        self.outputs = np.ascontiguousarray(np.asarray(outputs, dtype=np.uint32).reshape(-1, 2))

    def c(self):
        st = OrCircuit(self.n, self.gates.shape[0], _ptr(self.gates, U32P),
                       self.outputs.shape[0], _ptr(self.outputs, U32P))
        st._keep = (self.gates, self.outputs)
        return st


def eval_scalar(circ, bits):
    L = lib()
    inp = np.ascontiguousarray(np.asarray(bits, dtype=np.uint8))
    out = np.zeros(circ.outputs.shape[0], dtype=np.uint8)
    c = circ.c()
    assert L.or_eval_scalar(C.byref(c), _ptr(inp, U8P), _ptr(out, U8P)) == 0
    return out


def eval_words(circ, words):
    L = lib()
    inp = np.ascontiguousarray(np.asarray(words, dtype=np.uint64))
    out = np.zeros(circ.outputs.shape[0], dtype=np.uint64)
    c = circ.c()
    assert L.or_eval_words(C.byref(c), _ptr(inp, U64P), _ptr(out, U64P)) == 0
    return out


def sat_range(circ, begin=0, end=None, threads=0):
    """(count, lowest or None) over natural-order indices [begin, end)."""
    L = lib()
    if end is None:
        end = 1 << circ.n
    cnt, low = C.c_uint64(), C.c_uint64()
    c = circ.c()
    rc = L.or_sat_range(C.byref(c), begin, end, threads, C.byref(cnt), C.byref(low))
    assert rc == 0, rc
    return cnt.value, (None if low.value == 0xFFFFFFFFFFFFFFFF else low.value)


class QuantReducer:
    """Restatement of qsat.rs QuantReducer; quants is a string of 'A'/'E'."""

    def __init__(self, quants):
        q = np.array([1 if ch in "Aa" else 0 for ch in quants], dtype=np.uint8)
        self._h = lib().or_qr_new(_ptr(q, U8P), len(q))
        assert self._h

    def push(self, index, item):
        assert lib().or_qr_push(self._h, index, int(bool(item))) == 0

    def push_words(self, words, first=0):
        """Items of packed 32-bit words (item first + k = bit k%32 of word
        k/32), in index order from `first`."""
        w = np.ascontiguousarray(np.asarray(words, dtype=np.uint32))
        assert lib().or_qr_push_words_from(self._h, first, _ptr(w, U32P), len(w)) == 0

    def final_result(self):
        rv, sb, hs, sol = C.c_int(), C.c_uint32(), C.c_int(), C.c_uint64()
        if not lib().or_qr_final(self._h, C.byref(rv), C.byref(sb), C.byref(hs), C.byref(sol)):
            return None
        return {"reversed": bool(rv.value), "solution_bits": sb.value,
                "solution": sol.value if hs.value else None}

    def __del__(self):
        if getattr(self, "_h", None):
            lib().or_qr_free(self._h)
            self._h = None


def qsat(circ, quants, mode=1, threads=0):
    L = lib()
    q = np.array([1 if ch in "Aa" else 0 for ch in quants], dtype=np.uint8)
    assert len(q) == circ.n
    rv, sb, hs, sol = C.c_int(), C.c_uint32(), C.c_int(), C.c_uint64()
    c = circ.c()
    rc = L.or_qsat(C.byref(c), _ptr(q, U8P), mode, threads, C.byref(rv), C.byref(sb),
                   C.byref(hs), C.byref(sol))
    assert rc == 0, rc
    return {"reversed": bool(rv.value), "solution_bits": sb.value,
            "solution": sol.value if hs.value else None}


def stop_table(circ, threads=0):
    L = lib()
    t = np.zeros(1 << circ.n, dtype=np.uint64)
    c = circ.c()
    assert L.or_stop_table(C.byref(c), threads, _ptr(t, U64P)) == 0
    return t


def stop_solve(n, u, table, mode=0, threads=0):
    L = lib()
    t = np.ascontiguousarray(table, dtype=np.uint64)
    found, st, en, steps, rounds = C.c_int(), C.c_uint64(), C.c_uint64(), C.c_uint64(), C.c_uint32()
    rc = L.or_stop_solve(n, u, _ptr(t, U64P), mode, threads, C.byref(found), C.byref(st),
                         C.byref(en), C.byref(steps), C.byref(rounds))
    assert rc == 0, rc
    if not found.value:
        return None
    return {"start": st.value, "end": en.value, "steps": steps.value, "rounds": rounds.value}


def stop_replay(circ, start, max_steps):
    L = lib()
    en, steps = C.c_uint64(), C.c_uint64()
    c = circ.c()
    r = L.or_stop_replay(C.byref(c), start, max_steps, C.byref(en), C.byref(steps))
    assert r >= 0
    return (en.value, steps.value) if r == 1 else None


def memimage_get(data, state_len, i):
    return lib().or_memimage_get(_ptr(data, U64P), state_len, i)


def memimage_set(data, state_len, i, value):
    lib().or_memimage_set(_ptr(data, U64P), state_len, i, value & 0xFFFFFFFFFFFFFFFF)


def greedy_partitioned(n, unknowns, table, partitions):
    """Partitioned greedysatostop on the table (or_greedy_partitioned)."""
    t = np.ascontiguousarray(table, dtype=np.uint64)
    st, en = C.c_uint64(), C.c_uint64()
    stage, part = C.c_uint32(), C.c_uint32()
    r = lib().or_greedy_partitioned(_ptr(t, U64P), n, unknowns, partitions, C.byref(st), C.byref(en),
                                    C.byref(stage), C.byref(part))
    assert r >= 0, r
    if r == 0:
        return None
    return {"start": st.value, "end": en.value, "stage": stage.value, "partition": part.value}


def memimage_find_solution(data, state_len, start, length, unknowns):
    s, e = C.c_uint64(), C.c_uint64()
    r = lib().or_memimage_find_solution(_ptr(data, U64P), state_len, start, length, unknowns,
                                        C.byref(s), C.byref(e))
    assert r >= 0
    return {"start": s.value, "end": e.value} if r == 1 else None

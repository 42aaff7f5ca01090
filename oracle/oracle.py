"""Python access to the CPU oracle -- TEST INFRASTRUCTURE ONLY.

Loaded by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg to
check (or time) the CUDA product against a scalar C++ restatement of the
reference (oracle/clast_oracle.cpp), and against the reference itself built
for the CPU (oracle/build_ref.py -> oracle/_ref/clast_ref) when present.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB = os.path.join(HERE, "libclast_oracle.so")
CLI = os.path.join(HERE, "clast_oracle")
REF = os.path.join(HERE, "_ref", "clast_ref")

FIELDS = ("t_id", "t_idx", "q_id", "q_idx", "t_len", "q_len", "match", "score", "evalue")
STAGE_RAW, STAGE_FILTERED, STAGE_ALIGNED, STAGE_FINAL = 1, 2, 3, 4


class _params(C.Structure):
    _fields_ = [("lmer", C.c_int32), ("stride", C.c_int32), ("cut_repeat", C.c_int32), ("width", C.c_int32),
                ("gap", C.c_int32), ("local", C.c_int32), ("cutoff", C.c_double), ("total_db", C.c_double),
                ("K", C.c_double), ("lambda_", C.c_double)]


class _hits(C.Structure):
    _fields_ = [("n", C.c_int64)] + [(f, C.POINTER(C.c_int32)) for f in FIELDS[:-1]] + \
               [("evalue", C.POINTER(C.c_double))]


_lib = None


def build():
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB):
            build()
        L = C.CDLL(LIB)
        L.oracle_window_search.restype = C.c_int
        L.oracle_window_search.argtypes = [C.POINTER(_params), C.c_char_p, C.c_int64, C.c_void_p, C.c_void_p,
                                           C.c_int32, C.c_int32, C.c_char_p, C.c_int64, C.c_void_p, C.c_void_p,
                                           C.c_int32, C.c_int32, C.c_int32, C.POINTER(_hits)]
        L.oracle_hits_free.argtypes = [C.POINTER(_hits)]
        L.oracle_main.restype = C.c_int
        L.oracle_main.argtypes = [C.c_int, C.POINTER(C.c_char_p), C.c_int]
        L.oracle_last_error.restype = C.c_char_p
        _lib = L
    return _lib


def window_search(s, t_bases: bytes, t_gw, t_len, t_begin: int, q_bases: bytes, q_gw, q_len, q_begin: int,
                  stage: int = STAGE_FINAL) -> dict:
    """Oracle result for one (target window, query window) pair; ``s`` has the
    fields of clast_b200.api.Setting."""
    L = lib()
    p = _params(s.lmer, s.stride, s.cut_repeat, s.width, s.gap, s.local, float(s.cutoff), float(s.total_db),
                float(s.K), float(s.lambda_))
    tg = np.ascontiguousarray(t_gw, dtype=np.int32)
    tl = np.ascontiguousarray(t_len, dtype=np.int32)
    qg = np.ascontiguousarray(q_gw, dtype=np.int32)
    ql = np.ascontiguousarray(q_len, dtype=np.int32)
    h = _hits()
    rc = L.oracle_window_search(C.byref(p), t_bases, len(t_bases), tg.ctypes.data, tl.ctypes.data, len(tg),
                                t_begin, q_bases, len(q_bases), qg.ctypes.data, ql.ctypes.data, len(qg), q_begin,
                                stage, C.byref(h))
    if rc != 0:
        raise RuntimeError("oracle error %d: %s" % (rc, L.oracle_last_error().decode()))
    try:
        n = int(h.n)
        out = {}
        for f in FIELDS:
            dt = np.float64 if f == "evalue" else np.int32
            out[f] = np.ctypeslib.as_array(getattr(h, f), shape=(n,)).astype(dt, copy=True) if n else np.zeros(0, dt)
        return out
    finally:
        L.oracle_hits_free(C.byref(h))


def run_cli(argv, threads: int = 0):
    """The oracle's whole command line in-process: (exit code, message)."""
    L = lib()
    args = ["clast_oracle"] + [str(a) for a in argv]
    arr = (C.c_char_p * len(args))(*[a.encode() for a in args])
    rc = L.oracle_main(len(args), arr, threads)
    return rc, (L.oracle_last_error().decode() if rc else "")


def ref_available() -> bool:
    return os.path.exists(REF)


def run_ref(argv, timeout=600):
    """The reference itself (built for the CPU by oracle/build_ref.py)."""
    r = subprocess.run([REF] + [str(a) for a in argv], capture_output=True, text=True, timeout=timeout)
    return r.returncode, r.stdout + r.stderr

"""
ctypes front end of oracle/_ref/libref_xpu.so (PG-Strom's expression
library host-compiled from the reference sources plus ref_harness.cpp).
TEST INFRASTRUCTURE ONLY.
"""
import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_ref", "libref_xpu.so")
_LIB = None


def available():
    return os.path.exists(SO)


def source_dir():
    """PG-Strom's src/ directory the library was built from (recorded by
    oracle/Makefile "ref"), or None."""
    rec = os.path.join(HERE, "_ref", "pgstrom_src.txt")
    if not os.path.exists(rec):
        return None
    with open(rec) as f:
        path = f.read().strip()
    return path if os.path.isdir(path) else None


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(SO)
        P = ctypes.c_void_p
        L.ref_hash_any.argtypes = [P, ctypes.c_int]
        L.ref_hash_any.restype = ctypes.c_uint32
        L.ref_numeric_decode.argtypes = [P, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int),
                                         ctypes.POINTER(ctypes.c_uint64), ctypes.POINTER(ctypes.c_uint64)]
        L.ref_open.argtypes = [P, ctypes.c_uint64, P, ctypes.c_char_p, ctypes.c_int]
        L.ref_open.restype = P
        L.ref_exec.argtypes = [P, P, ctypes.c_char_p, ctypes.c_int]
        L.ref_result.argtypes = [P, ctypes.c_char_p, ctypes.c_uint64]
        L.ref_result.restype = ctypes.c_uint64
        L.ref_close.argtypes = [P]
        L.ref_counts.argtypes = [P, ctypes.POINTER(ctypes.c_uint64)]
        _LIB = L
    return _LIB


def hash_any(data: bytes) -> int:
    a = np.frombuffer(data, dtype=np.uint8).copy() if data else np.zeros(1, dtype=np.uint8)
    return lib().ref_hash_any(ctypes.c_void_p(a.ctypes.data), len(data))


def numeric_decode(vl: bytes):
    a = np.frombuffer(vl, dtype=np.uint8).copy()
    k, w = ctypes.c_int(), ctypes.c_int()
    lo, hi = ctypes.c_uint64(), ctypes.c_uint64()
    if lib().ref_numeric_decode(ctypes.c_void_p(a.ctypes.data), ctypes.byref(k), ctypes.byref(w),
                                ctypes.byref(lo), ctypes.byref(hi)):
        return None
    v = (hi.value << 64) | lo.value
    if v >= 1 << 127:
        v -= 1 << 128
    return k.value, w.value, v


def run_counts(session: bytes, chunks, kmrels=None):
    """Runs the reference functions over the chunks; returns the row
    counters only (no groups written out)."""
    sess = np.frombuffer(session + b"\0" * 64, dtype=np.uint8).copy()
    km = kmrels.copy() if kmrels is not None else None
    err = ctypes.create_string_buffer(256)
    h = lib().ref_open(ctypes.c_void_p(sess.ctypes.data), len(session),
                       ctypes.c_void_p(km.ctypes.data) if km is not None else None, err, 256)
    if not h:
        raise RuntimeError("ref_open: " + err.value.decode())
    try:
        for ch in chunks:
            if lib().ref_exec(h, ctypes.c_void_p(ch.ctypes.data), err, 256):
                raise RuntimeError("ref_exec: " + err.value.decode())
        out = (ctypes.c_uint64 * 3)()
        lib().ref_counts(h, out)
        return {"nitems_raw": out[0], "nitems_in": out[1], "nitems_out": out[2]}
    finally:
        lib().ref_close(h)


def run(session: bytes, chunks, kmrels=None):
    """Runs the reference functions over the chunks; returns parsed JSON."""
    sess = np.frombuffer(session + b"\0" * 64, dtype=np.uint8).copy()
    km = kmrels.copy() if kmrels is not None else None
    err = ctypes.create_string_buffer(256)
    h = lib().ref_open(ctypes.c_void_p(sess.ctypes.data), len(session),
                       ctypes.c_void_p(km.ctypes.data) if km is not None else None, err, 256)
    if not h:
        raise RuntimeError("ref_open: " + err.value.decode())
    try:
        for ch in chunks:
            if lib().ref_exec(h, ctypes.c_void_p(ch.ctypes.data), err, 256):
                raise RuntimeError("ref_exec: " + err.value.decode())
        n = lib().ref_result(h, None, 0)
        buf = ctypes.create_string_buffer(n)
        lib().ref_result(h, buf, n)
        return json.loads(buf.value.decode())
    finally:
        lib().ref_close(h)

"""
ctypes front end of oracle/_ref/libref_gpu.so: PG-Strom's own device
executor kern_gpujoin_main, built for sm_100a from the reference sources
(oracle/_ref/pgstrom_sm100a.fatbin, oracle/Makefile "ref_gpu"), launched the
way PG-Strom's GPU service launches it (ref_gpu.cpp).  TEST INFRASTRUCTURE
ONLY: the reference kernel as a checker and as the GPU-to-GPU baseline.
"""
import ctypes
import json
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
SO = os.path.join(HERE, "_ref", "libref_gpu.so")
FATBIN = os.path.join(HERE, "_ref", "pgstrom_sm100a.fatbin")
_LIB = None


def available():
    return os.path.exists(SO) and os.path.exists(FATBIN)


def lib():
    global _LIB
    if _LIB is None:
        L = ctypes.CDLL(SO)
        P, S, E = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_char_p
        L.rg_open.argtypes = [ctypes.c_char_p, ctypes.c_int, E, S]
        L.rg_open.restype = ctypes.c_int
        L.rg_session.argtypes = [P, S, P, S, S, E, S]
        L.rg_session.restype = P
        L.rg_exec.argtypes = [P, ctypes.POINTER(ctypes.c_uint64), ctypes.c_uint32,
                              ctypes.POINTER(ctypes.c_double), E, S]
        L.rg_exec.restype = ctypes.c_int
        L.rg_final.argtypes = [P, P, S, E, S]
        L.rg_final.restype = ctypes.c_int64
        L.rg_info.argtypes = [P, E, S]
        L.rg_close.argtypes = [P]
        L.rg_upload.argtypes = [P, S]
        L.rg_upload.restype = ctypes.c_uint64
        L.rg_free.argtypes = [ctypes.c_uint64]
        _LIB = L
    return _LIB


class RefError(RuntimeError):
    pass


def open_device(dindex=0):
    err = ctypes.create_string_buffer(512)
    if lib().rg_open(FATBIN.encode(), dindex, err, 512):
        raise RefError("rg_open: " + err.value.decode())


def upload(arr):
    """A device copy of a chunk for the reference kernel (it stamps t_ctid
    into heap pages, so it gets copies of its own)."""
    a = np.ascontiguousarray(arr)
    d = lib().rg_upload(ctypes.c_void_p(a.ctypes.data), a.nbytes)
    if not d:
        raise RefError("rg_upload failed")
    return d


def free(d):
    lib().rg_free(d)


class RefSession:
    """One query on the reference kernel: the session blob and the inner
    relations (kern_multirels) as the CUDA path receives them."""

    def __init__(self, session: bytes, kmrels=None, final_min=0):
        s = np.frombuffer(bytes(session), dtype=np.uint8).copy()
        km = np.ascontiguousarray(kmrels) if kmrels is not None else None
        err = ctypes.create_string_buffer(512)
        self.h = lib().rg_session(ctypes.c_void_p(s.ctypes.data), s.nbytes,
                                  ctypes.c_void_p(km.ctypes.data) if km is not None else None,
                                  km.nbytes if km is not None else 0, final_min, err, 512)
        if not self.h:
            raise RefError("rg_session: " + err.value.decode())

    def exec(self, dptrs):
        """One task per chunk (device addresses from upload()), in order;
        returns the device milliseconds from the first launch to the end of
        the last (the per-chunk synchronisations between them included)."""
        a = (ctypes.c_uint64 * len(dptrs))(*dptrs)
        ms = ctypes.c_double()
        err = ctypes.create_string_buffer(512)
        rc = lib().rg_exec(self.h, a, len(dptrs), ctypes.byref(ms), err, 512)
        if rc:
            raise RefError("rg_exec: " + err.value.decode())
        return ms.value

    def final(self):
        err = ctypes.create_string_buffer(512)
        n = lib().rg_final(self.h, None, 0, err, 512)
        if n < 0:
            raise RefError("rg_final: " + err.value.decode())
        out = np.zeros(max(n, 8), dtype=np.uint8)
        if lib().rg_final(self.h, ctypes.c_void_p(out.ctypes.data), out.nbytes, err, 512) < 0:
            raise RefError("rg_final: " + err.value.decode())
        return out[:n]

    def info(self):
        buf = ctypes.create_string_buffer(1024)
        lib().rg_info(self.h, buf, 1024)
        return json.loads(buf.value.decode())

    def close(self):
        if self.h:
            lib().rg_close(self.h)
            self.h = None

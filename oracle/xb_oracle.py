"""
ctypes front end of the CPU oracle (liboracle.so).  TEST INFRASTRUCTURE
ONLY: used by tests/, __graft_entry__.smoke() and bench.py's cpu_baseline
leg as the checker; the product never imports it.
"""
import ctypes
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None


def lib():
    global _LIB
    if _LIB is None:
        so = os.path.join(HERE, "liboracle.so")
        src = os.path.join(HERE, "xb_oracle.c")
        if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
            subprocess.run(["make", "-s", "-C", HERE, "liboracle.so"], check=True)
        L = ctypes.CDLL(so)
        P, U64 = ctypes.c_void_p, ctypes.c_uint64
        L.xo_open.argtypes = [P, U64, P, U64, ctypes.POINTER(P), ctypes.c_char_p, ctypes.c_int]
        L.xo_exec.argtypes = [P, P, ctypes.c_char_p, ctypes.c_int]
        L.xo_stats.argtypes = [P, ctypes.POINTER(ctypes.c_uint64)]
        L.xo_final.argtypes = [P, P, U64]
        L.xo_final.restype = ctypes.c_uint64
        L.xo_close.argtypes = [P]
        L.xo_proj_rows.argtypes = [P, P, U64, ctypes.POINTER(U64), ctypes.POINTER(U64)]
        L.xo_proj_rows.restype = ctypes.c_uint64
        L.xo_proj_reset.argtypes = [P]
        L.xo_hash_bytes.argtypes = [P, ctypes.c_uint32]
        L.xo_hash_bytes.restype = ctypes.c_uint32
        _LIB = L
    return _LIB


def _p(a):
    return ctypes.c_void_p(a.ctypes.data) if a is not None else None


class Oracle:
    def __init__(self, session: bytes, kmrels=None):
        self._session = np.frombuffer(session, dtype=np.uint8).copy()
        self._kmrels = kmrels
        self.h = ctypes.c_void_p()
        err = ctypes.create_string_buffer(256)
        rc = lib().xo_open(_p(self._session), self._session.nbytes, _p(kmrels),
                           kmrels.nbytes if kmrels is not None else 0, ctypes.byref(self.h), err, 256)
        if rc:
            raise RuntimeError(err.value.decode())

    def exec(self, kds: np.ndarray):
        err = ctypes.create_string_buffer(256)
        if lib().xo_exec(self.h, _p(kds), err, 256):
            raise RuntimeError("oracle: " + err.value.decode())

    def stats(self):
        s = (ctypes.c_uint64 * 12)()
        lib().xo_stats(self.h, s)
        return {"nitems_raw": s[0], "nitems_in": s[1], "nitems_out": s[2],
                "depth_out": [s[3 + i] for i in range(8)]}

    def final(self):
        n = lib().xo_final(self.h, None, 0)
        if n == 0:
            return None
        buf = np.zeros(n, dtype=np.uint8)
        lib().xo_final(self.h, _p(buf), n)
        return buf

    def proj_rows(self, reset=False):
        """Projected rows since the last reset: (list of tuple images with
        the row id cut off, kds_dst usage the rows take)."""
        n, usage = ctypes.c_uint64(), ctypes.c_uint64()
        nb = lib().xo_proj_rows(self.h, None, 0, ctypes.byref(n), ctypes.byref(usage))
        buf = np.zeros(max(nb, 8), dtype=np.uint8)
        lib().xo_proj_rows(self.h, _p(buf), nb, ctypes.byref(n), ctypes.byref(usage))
        rows, pos = [], 0
        for _ in range(n.value):
            t_len = int(buf[pos:pos + 4].view(np.uint32)[0])
            rows.append(bytes(buf[pos:pos + t_len - 4]))
            pos += (t_len + 7) & ~7
        if reset:
            lib().xo_proj_reset(self.h)
        return rows, usage.value

    def close(self):
        if self.h:
            lib().xo_close(self.h)
            self.h = ctypes.c_void_p()


def hash_bytes(data: bytes) -> int:
    a = np.frombuffer(data, dtype=np.uint8).copy() if data else np.zeros(1, dtype=np.uint8)
    return lib().xo_hash_bytes(_p(a), len(data))

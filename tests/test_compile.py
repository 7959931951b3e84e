"""OpenSession-time translation of the session bytecode (xb_compile.cpp),
on the CPU: a session the backend sent broken is refused with a message
(the reference's OpenSession answers such sessions with an error, never a
crash of the GPU service), and sessions with random bytes changed are
either translated or refused, never crash the process."""
import ctypes
import os
import struct
import subprocess
import sys

import pytest

import xb_configs as C
import xpu_b200

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def _lib():
    if not os.path.exists(xpu_b200.LIB_PATH):
        pytest.skip("library not built")
    return ctypes.CDLL(xpu_b200.LIB_PATH)


def compile_session(sess, km=None, size=None):
    L = _lib()
    sb = bytes(sess)
    kb = bytes(km) if km is not None else None
    plan = ctypes.create_string_buffer(1 << 20)
    err = ctypes.create_string_buffer(1024)
    rc = L.xb_compile_session(sb, ctypes.c_size_t(len(sb) if size is None else size), ctypes.c_uint64(1 << 32),
                              kb, plan, err, ctypes.c_size_t(len(err)))
    return rc, err.value.decode(errors="replace")


def _scan():
    _, sess, _, _, _ = C.scan_groupby(nrows=100)
    return bytearray(bytes(sess))


def test_valid_session_translates():
    assert compile_session(_scan()) == (0, "")


def test_truncated_session_is_refused():
    rc, msg = compile_session(_scan(), size=64)
    assert rc != 0 and "shorter than kern_session_info" in msg


def test_slot_descriptors_outside_the_session_are_refused():
    s = _scan()
    struct.pack_into("<I", s, 16, len(s) - 4)               # kcxt_kvars_defs near the end
    rc, msg = compile_session(s)
    assert rc != 0 and "out of the session" in msg


def test_expression_offset_outside_the_session_is_refused():
    s = _scan()
    struct.pack_into("<I", s, 56, len(s) + 64)              # xpucode_scan_quals past the end
    rc, msg = compile_session(s)
    assert rc != 0 and "out of the session" in msg


def test_broken_expression_header_is_refused():
    s = _scan()
    quals, = struct.unpack_from("<I", s, 56)
    assert quals != 0
    t = bytearray(s)
    struct.pack_into("<I", t, quals, 8)                     # kern_expression.len too short
    rc, msg = compile_session(t)
    assert rc != 0 and "length" in msg and "broken" in msg
    t = bytearray(s)
    kexp_len, = struct.unpack_from("<I", t, quals)
    t[quals + kexp_len - 1] ^= 0xff                         # the trailing magic word
    rc, msg = compile_session(t)
    assert rc != 0 and "magic mismatch" in msg


FUZZ = r'''
import ctypes, sys
import numpy as np
sys.path[:0] = sys.argv[4:]
import xb_configs as C, xpu_b200
L = ctypes.CDLL(xpu_b200.LIB_PATH)
which, seed, n = sys.argv[1], int(sys.argv[2]), int(sys.argv[3])
if which == "scan":
    _, s, k, _, _ = C.scan_groupby(nrows=100)
elif which == "wide":
    _, s, k, _, _ = C.wide_groupby(nrows=100, ngroups=10)
elif which == "join":
    _, s, k, _, _ = C.join_groupby(nfact=100, ndim1=50, ndim2=10)
elif which == "projection":
    _, s, k, _ = C.join_projection(nfact=100, ndim1=50, ndim2=10)
else:
    _, s, _, _ = C.arrow_nulls(nrows=100, nkeys=10, rows_per_chunk=100)
    k = None
s = bytes(s)
kb = bytes(k) if k is not None else None
r = np.random.default_rng(seed)
plan = ctypes.create_string_buffer(1 << 20)
err = ctypes.create_string_buffer(1024)
done = 0
for _ in range(n):
    t = bytearray(s)
    for _ in range(int(r.integers(1, 4))):
        pos = int(r.integers(0, len(t)))
        t[pos] = int(r.integers(0, 256)) if r.random() < 0.5 else t[pos] ^ (1 << int(r.integers(0, 8)))
    L.xb_compile_session(bytes(t), ctypes.c_size_t(len(t)), ctypes.c_uint64(1 << 32), kb, plan, err,
                         ctypes.c_size_t(1024))
    done += 1
print(done)
'''


@pytest.mark.parametrize("which", ["scan", "wide", "join", "projection", "arrow"])
def test_mutated_sessions_never_crash(which):
    """1,500 sessions with one to three bytes changed at random, each
    translated or refused; the translating process must finish (a crash
    ends the child process, not the test)."""
    paths = [os.path.join(ROOT, "pg-strom_b200"), os.path.join(ROOT, "pg-strom_b200", "producer"),
             os.path.join(ROOT, "oracle")]
    _lib()
    r = subprocess.run([sys.executable, "-c", FUZZ, which, "7", "1500"] + paths,
                       capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.split()[-1] == "1500"

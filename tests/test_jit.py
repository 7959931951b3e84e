"""The session-specialised kernels: the source generated for each workload's
translated session compiles for sm_100a with NVRTC.  Compilation needs no
GPU; the kernels' results are checked against the oracle by the GPU parity
tests (test_gpu_parity.py runs every case on both kernels)."""
import ctypes
import os

import pytest

import xb_configs as C
import xpu_b200

PLAN_BYTES = 1 << 20


def _lib():
    if not os.path.exists(xpu_b200.LIB_PATH):
        pytest.skip("library not built")
    return ctypes.CDLL(xpu_b200.LIB_PATH)


def _translate(L, sess, km):
    sb = bytes(sess)
    kb = bytes(km) if km is not None else None
    plan = ctypes.create_string_buffer(PLAN_BYTES)
    err = ctypes.create_string_buffer(1024)
    rc = L.xb_compile_session(sb, ctypes.c_size_t(len(sb)), ctypes.c_uint64(1 << 32), kb, plan, err,
                              ctypes.c_size_t(len(err)))
    assert rc == 0, err.value.decode()
    return plan


def _session(case):
    if case == "scan_groupby":
        _, s, _, _, _ = C.scan_groupby(nrows=1000)
        return s, None, ord("b")
    if case in ("join_groupby", "join_groupby_row"):
        _, s, k, _, _ = C.join_groupby(nfact=1000, ndim1=100, ndim2=10)
        return s, k, ord("b" if case == "join_groupby" else "r")
    if case == "arrow_groupby":
        _, s, _, _ = C.arrow_groupby(nrows=1000, nkeys=100, rows_per_chunk=1000, with_expect=False)
        return s, None, ord("a")
    if case == "wide_groupby":
        _, s, _, _, _ = C.wide_groupby(nrows=1000, ngroups=50)
        return s, None, ord("b")
    if case == "scan_nogroup":
        _, s, _, _, _ = C.scan_nogroup(nrows=1000)
        return s, None, ord("b")
    if case == "long_varlena":
        _, s, _, _, _ = C.long_varlena_groupby(nrows=1000)
        return s, None, ord("b")
    if case == "arrow_nulls":
        _, s, _, _ = C.arrow_nulls(nrows=1000, nkeys=50, rows_per_chunk=1000)
        return s, None, ord("a")
    if case == "scan_projection":
        _, s, _, _ = C.scan_projection(nrows=1000)
        return s, None, ord("b")
    if case == "join_projection":
        _, s, k, _ = C.join_projection(nfact=1000, ndim1=100, ndim2=10)
        return s, k, ord("b")
    if case == "arrow_int2_bool":
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            _, s, _, _ = C.arrow_int2_bool(d, nrows=1000)
        return s, None, ord("a")
    raise ValueError(case)


CASES = ["scan_groupby", "join_groupby", "arrow_groupby", "join_groupby_row", "wide_groupby",
         "scan_nogroup", "long_varlena", "arrow_nulls", "scan_projection", "join_projection", "arrow_int2_bool"]


@pytest.mark.parametrize("name", CASES)
def test_specialised_kernel_compiles(name):
    L = _lib()
    sess, km, fmt = _session(name)
    plan = _translate(L, sess, km)
    nbytes = ctypes.c_uint64(0)
    ms = ctypes.c_double(0.0)
    err = ctypes.create_string_buffer(2048)
    rc = L.xb_jit_check(plan, ctypes.c_uint32(fmt), ctypes.byref(nbytes), ctypes.byref(ms), err,
                        ctypes.c_size_t(len(err)))
    msg = err.value.decode()
    if rc != 0 and "libnvrtc" in msg:
        pytest.skip(msg)
    assert rc == 0, f"{name}: {msg}"
    assert nbytes.value > 0


def _walk_plan(L):
    """the plain scan session's plan with the heap layout of its table
    noted (numeric c before the group key g: no fixed offsets, a walk)"""
    tbl, sess, _, _, _ = C.scan_groupby(nrows=1000)
    plan = _translate(L, sess, None)
    head = bytes(tbl.kds_header("b"))
    L.xb_plan_note_layout(plan, head)
    return plan


def test_walk_kernel_compiles():
    L = _lib()
    plan = _walk_plan(L)
    n = ctypes.c_size_t(0)
    buf = ctypes.create_string_buffer(1 << 21)
    assert L.xb_jit_source(plan, ctypes.c_uint32(ord("b")), buf, ctypes.c_size_t(len(buf)), ctypes.byref(n)) == 0
    src = buf.value.decode()
    # columns 1..5 walked; the numeric column's varlena header read, nullmap tested
    assert "xbj_walk(" in src and "/* column 4: attlen -1, attalign 4 */" in src
    assert "(nullmap[0] >> 2) & 1" in src and "#define XBJ_LAY_FIXED 0" in src
    nbytes = ctypes.c_uint64(0)
    ms = ctypes.c_double(0.0)
    err = ctypes.create_string_buffer(2048)
    rc = L.xb_jit_check(plan, ctypes.c_uint32(ord("b")), ctypes.byref(nbytes), ctypes.byref(ms), err,
                        ctypes.c_size_t(len(err)))
    msg = err.value.decode()
    if rc != 0 and "libnvrtc" in msg:
        pytest.skip(msg)
    assert rc == 0, msg


def test_generated_source_names_the_plan():
    L = _lib()
    _, sess, km, _, _ = C.join_groupby(nfact=1000, ndim1=100, ndim2=10)
    plan = _translate(L, sess, km)
    n = ctypes.c_size_t(0)
    buf = ctypes.create_string_buffer(1 << 20)
    assert L.xb_jit_source(plan, ctypes.c_uint32(ord("b")), buf, ctypes.c_size_t(len(buf)), ctypes.byref(n)) == 0
    src = buf.value.decode()
    assert n.value == len(src)
    # two join depths, a group-by and no interpreter loop
    assert "/* depth 1 */" in src and "/* depth 2 */" in src and "/* depth 3 */" not in src
    assert "xbj_group_get<true>" in src and "xb_vm_exec" not in src

"""Device projection (rows written as kern_tupitems into a KDS_FORMAT_ROW
kds_dst): the oracle's rows pinned against the generators' column arrays,
and the specialised kernel's source compiling for projection sessions.
The GPU parity of the same workloads is in test_gpu_projection.py."""
import ctypes
import struct

import numpy as np
import pytest

import xb_configs as C
import xb_oracle as O
import xb_rows as RW


def _dst_columns(sess):
    off, = struct.unpack_from("<I", sess, 128)
    return RW.kds_columns(sess[off:])


def _oracle_rows(sess, chunks, kmrels=None):
    o = O.Oracle(sess, kmrels)
    for ch in chunks:
        o.exec(ch)
    rows, usage = o.proj_rows()
    st = o.stats()
    o.close()
    return rows, usage, st


@pytest.mark.parametrize("margin", [0, 24])
def test_oracle_scan_projection(margin):
    tbl, sess, expect, meta = C.scan_projection(nrows=30_000, htup_margin=margin)
    rows, usage, st = _oracle_rows(sess, tbl.block_chunks(pages_per_chunk=64))
    assert st["nitems_in"] == meta["nitems_in"] == len(rows) == len(expect)
    cols = _dst_columns(sess)
    blob, offs = tbl.col("c").values
    seen = set()
    total = 0
    for img in rows:
        v = RW.decode_tuple(img + b"\0" * 4, 0, cols)
        rid = v[0]
        assert (v[1], v[2], v[4]) == expect[rid]
        assert v[3] == bytes(blob[offs[rid]:offs[rid + 1]])      # numeric varlena as stored
        seen.add(rid)
        t_len = len(img) + 4
        total += (((t_len + 7) & ~7) + margin + 7) & ~7
    assert seen == set(expect)
    assert usage == total


def test_oracle_scan_projection_null_bitmap():
    tbl, sess, expect, _ = C.scan_projection(nrows=8_000, null_frac=0.5)
    rows, _, _ = _oracle_rows(sess, tbl.block_chunks(pages_per_chunk=32))
    n_null = 0
    for img in rows:
        im, = struct.unpack_from("<H", img, 12)
        t_hoff = img[14]
        v = RW.decode_tuple(img + b"\0" * 4, 0, _dst_columns(sess))
        if v[2] is None:
            n_null += 1
            assert im & RW.HEAP_HASNULL and img[15] == 0b11011 and t_hoff == 8 + 16
        else:
            assert not im & RW.HEAP_HASNULL and t_hoff == 8 + 16
    assert n_null == sum(1 for e in expect.values() if e[1] is None) > 0


@pytest.mark.parametrize("copies,stride,miss", [(1, 1, 0.0), (3, 7, 0.2)])
def test_oracle_join_projection(copies, stride, miss):
    fact, sess, km, meta = C.join_projection(nfact=20_000, dim1_copies=copies, key_stride=stride,
                                             miss_frac=miss)
    rows, _, st = _oracle_rows(sess, fact.block_chunks(pages_per_chunk=50), km)
    assert st["nitems_out"] == meta["nitems_out"] == len(rows)
    cols = _dst_columns(sess)
    got = sorted(tuple(RW.decode_tuple(img + b"\0" * 4, 0, cols)) for img in rows)
    assert got == meta["rows"]


def _compile_ok(sess, km):
    from test_jit import _lib, _translate
    L = _lib()
    plan = _translate(L, sess, km)
    nb, ms = ctypes.c_uint64(), ctypes.c_double()
    err = ctypes.create_string_buffer(8192)
    rc = L.xb_jit_check(plan, ctypes.c_uint32(ord("b")), ctypes.byref(nb), ctypes.byref(ms), err,
                        ctypes.c_size_t(len(err)))
    msg = err.value.decode(errors="replace")
    if rc != 0 and "libnvrtc" in msg:
        pytest.skip(msg)
    return rc, msg


def test_specialised_kernel_compiles_for_projection():
    tbl, sess, _, _ = C.scan_projection(nrows=1000)
    rc, msg = _compile_ok(sess, None)
    assert rc == 0, msg
    fact, sess2, km, _ = C.join_projection(nfact=1000)
    rc, msg = _compile_ok(sess2, km)
    assert rc == 0, msg


def test_oracle_pinned_inner_projection():
    # a scan of dim1 projecting (pk, region) rows that carry HashValue(pk):
    # the hash is the join's inner hash, the values the dim1 columns
    fact, sess, km, expect, meta = C.join_groupby(nfact=1000, ndim1=3000, ndim2=70)
    dims = meta["dims"]
    ps = C.pinned_dim1_session(nslots=1024)
    rows, usage, st = _oracle_rows(ps, dims["dim1"].block_chunks(pages_per_chunk=5))
    assert len(rows) == 3000
    cols = _dst_columns(ps)
    got = {}
    for img in rows:
        h, = struct.unpack_from("<I", img, 4)
        pk, region = RW.decode_tuple(img + b"\0" * 8, 0, cols)
        got[pk] = (h, region.decode())
    pk1 = dims["pk1"]
    want_h = C.host_join_hash_int4(pk1)
    assert sorted(got) == sorted(int(x) for x in pk1)
    for i, pk in enumerate(pk1.tolist()):
        assert got[pk][0] == int(want_h[i])

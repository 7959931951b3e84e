"""The C-ABI library loads and exports every entry point of include/*.h."""
import ctypes
import os
import re
import struct

import numpy as np

import xpu_b200

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = []
    for h in os.listdir(os.path.join(ROOT, "include")):
        if not h.endswith(".h"):
            continue
        src = open(os.path.join(ROOT, "include", h)).read()
        names += re.findall(r"^\s*(?:int|void|uint32_t)\s+(xpuB200\w+)\s*\(", src, re.M)
    return sorted(set(names))


def test_library_exports_declared_symbols():
    L = xpu_b200.lib()
    names = declared_symbols()
    assert len(names) >= 10
    for n in names:
        assert hasattr(L, n), n


def test_library_is_sm100a_build():
    data = open(xpu_b200.LIB_PATH, "rb").read()
    assert b"sm_100a" in data


def _kds_check(buf):
    L = xpu_b200.lib()
    L.xb_kds_check.argtypes = [ctypes.c_void_p, ctypes.POINTER(xpu_b200.KernErrorbuf)]
    L.xb_kds_check.restype = ctypes.c_int
    a = np.ascontiguousarray(buf)
    eb = xpu_b200.KernErrorbuf()
    rc = L.xb_kds_check(ctypes.c_void_p(a.ctypes.data), ctypes.byref(eb))
    return rc, eb.message.decode()


COLMETA, COLMETA_SZ = 72, 168


def test_chunk_checks_reject_broken_chunks():
    """The checks ExecTask applies to a chunk before any launch (no device
    needed): well-formed heap and Arrow chunks pass; a chunk whose pages or
    Arrow buffers lie outside its length, whose Arrow ranges wrap around
    2^64, whose columns outnumber their descriptors, or whose format is
    unknown is rejected with ERRCODE_DEVICE_ERROR and a message, so no
    kernel reads outside the chunk."""
    import xb_configs as C
    tbl, _, _, _, _ = C.scan_groupby(nrows=2_000)
    blk = tbl.block_chunks(pages_per_chunk=16)[0]
    assert _kds_check(blk) == (0, "")

    bad = blk.copy()
    struct.pack_into("<I", bad, 16, 10_000)                       # nitems: pages past the length
    rc, msg = _kds_check(bad)
    assert rc == ord("E") and "broken" in msg
    bad = blk.copy()
    struct.pack_into("<I", bad, 44, 64)                           # block_offset inside the header
    assert _kds_check(bad)[0] == ord("E")
    bad = blk.copy()
    bad[24] = ord("x")
    rc, msg = _kds_check(bad)
    assert rc == ord("E") and "unsupported KDS format" in msg

    chunks, _, _, _ = C.arrow_groupby(nrows=2_000, nkeys=100, rows_per_chunk=2_000, with_expect=False)
    arw = chunks[0]
    assert _kds_check(arw) == (0, "")
    ncols, = struct.unpack_from("<I", arw, 20)
    for field in (120, 136, 152):                                 # nullmap, values, extra
        bad = arw.copy()
        off = COLMETA + COLMETA_SZ * (ncols - 1) + field
        struct.pack_into("<QQ", bad, off, (1 << 64) - 8, 16)      # offset + length wraps to 8
        rc, msg = _kds_check(bad)
        assert rc == ord("E") and "out of the chunk" in msg, field
    bad = arw.copy()
    struct.pack_into("<I", bad, 68, ncols - 1)                    # nr_colmeta < ncols
    rc, msg = _kds_check(bad)
    assert rc == ord("E") and "column descriptors" in msg
    bad = arw.copy()
    values_offset, = struct.unpack_from("<Q", arw, COLMETA + 136)
    struct.pack_into("<Q", bad, COLMETA + 136, values_offset + 4)
    rc, msg = _kds_check(bad)
    assert rc == ord("E") and "aligned" in msg


def test_chunk_checks_row_index_inside_the_chunk():
    """A KDS_FORMAT_ROW source chunk: its row index (after the hash slots)
    must fit in the chunk's length for every one of its nitems rows."""
    import xb_configs as C
    tbl, _, _, _, _ = C.scan_groupby(nrows=100)
    head = bytes(tbl.kds_header("r", 10))
    buf = np.zeros(len(head) + 8 * 10 + 64, dtype=np.uint8)
    buf[:len(head)] = np.frombuffer(head, dtype=np.uint8)
    struct.pack_into("<Q", buf, 0, buf.nbytes)
    assert _kds_check(buf) == (0, "")
    struct.pack_into("<I", buf, 16, 19)                           # 19 rows: the index runs 8 bytes past
    rc, msg = _kds_check(buf)
    assert rc == ord("E") and "ROW chunk is broken" in msg
    struct.pack_into("<I", buf, 16, 10)
    assert _kds_check(buf) == (0, "")
    struct.pack_into("<I", buf, 40, 9)                            # 9 hash slots before the index
    assert _kds_check(buf)[0] == ord("E")
    for ch in tbl.row_chunks(rows_per_chunk=30):                  # chunks of the ROW producer
        assert _kds_check(ch) == (0, "")

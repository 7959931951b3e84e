"""Chunk producers over files (relscan.c / Arrow_Fdw counterparts): a heap
relation segment file read back into KDS_FORMAT_BLOCK chunks is the same
chunks, byte for byte, as the ones built in memory; an Arrow IPC file
with a dictionary-encoded text column becomes KDS_FORMAT_ARROW chunks the
oracle (and the device, test_gpu_files.py) group by that column."""
import numpy as np
import pytest

import xb_configs as C
import xb_files as XF
import xb_final as F
import xb_oracle as O
from xb_producer import Agg, Const, Func, SessionBuilder, Var, BoolOp


def test_heap_file_round_trip(tmp_path):
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=60_000, seed_config=30)
    path = str(tmp_path / "16384")
    nblocks = XF.write_heap_relation(tbl, path)
    mem = tbl.block_chunks(pages_per_chunk=200)
    got = XF.heap_file_chunks(tbl, path, pages_per_chunk=200)
    assert sum(int(np.frombuffer(c[16:20].tobytes(), np.uint32)[0]) for c in got) == nblocks
    assert len(got) == len(mem)
    for a, b in zip(got, mem):
        assert a.tobytes() == b.tobytes()
    o = O.Oracle(sess)
    for ch in got:
        o.exec(ch)
    truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
    assert F.compare_groups(F.decode_kds_final(o.final(), sess), truth) == []
    o.close()


WORDS = ["alpha", "bravo", "charlie", "delta", "echo-" * 30, "foxtrot", "golf", "hotel"]


def arrow_dict_case(tmp_path, nrows=40_000, seed=31):
    """An Arrow IPC file (k int8, v1 int4, v2 float8, d date, s text
    dictionary-encoded) and a GROUP BY s session with its expected groups."""
    r = np.random.default_rng(seed)
    k = r.integers(0, 1000, nrows, dtype=np.int64)
    v1 = r.integers(-1000, 1000, nrows, dtype=np.int32)
    v2 = r.lognormal(0.0, 1.0, nrows)
    d = np.datetime64("2015-01-01") + r.integers(0, 3652, nrows).astype("timedelta64[D]")
    codes = r.integers(0, len(WORDS), nrows)
    s = [WORDS[c] for c in codes]
    path = str(tmp_path / "t.arrow")
    XF.write_arrow_ipc(path, {"k": k, "v1": v1, "v2": v2, "d": d, "s": s}, dictionary={"s"},
                       batch_rows=15_000)
    lo, hi = 17532, 18262
    vv1, vv2, vd, vs = Var(0, 2, "int4"), Var(0, 3, "float8"), Var(0, 4, "date"), Var(0, 5, "text")
    sess = SessionBuilder(0, C.DEVTASK_PREAGG | C.DEVKIND_GPU).build(
        scan_quals=BoolOp("And", [Func("date_ge", [vd, Const("date", lo - C.UNIX_TO_PG_DAYS)], "bool"),
                                  Func("date_lt", [vd, Const("date", hi - C.UNIX_TO_PG_DAYS)], "bool")]),
        groupby_keys=[vs],
        aggs=[Agg("NROWS_ANY"), Agg("PSUM_INT", Func("int4_to_int8", [vv1], "int8")),
              Agg("PMIN_FP64", vv2), Agg("PMAX_FP64", vv2), Agg("PSUM_FP", vv2)],
        ngroups_estimate=16.0)
    days = (d - np.datetime64("1970-01-01")).astype(np.int64)
    m = (days >= lo) & (days < hi)
    expect = {}
    for c, w in enumerate(WORDS):
        sel = m & (codes == c)
        if not sel.any():
            continue
        x = v2[sel]
        fs = 0.0
        for t in x:
            fs += float(t)
        n = int(sel.sum())
        expect[(w.encode(),)] = [n, (n, int(v1[sel].astype(np.int64).sum())), (1, float(x.min())),
                                 (1, float(x.max())), (n, fs)]
    return path, sess, expect, int(m.sum())


def test_arrow_ipc_dictionary_column(tmp_path):
    path, sess, expect, nin = arrow_dict_case(tmp_path)
    chunks, tdef = XF.arrow_ipc_chunks(path)
    assert len(chunks) == 3 and [c.typ for c in tdef.columns] == ["int8", "int4", "float8", "date", "text"]
    o = O.Oracle(sess)
    for ch in chunks:
        o.exec(ch)
    assert o.stats()["nitems_in"] == nin
    assert F.compare_groups(F.decode_kds_final(o.final(), sess), expect) == []
    o.close()


def test_heap_file_iovec_matches_chunks(tmp_path):
    """the header plus the file pages an I/O vector names, laid out at
    base_offset + m_offset, are the chunk heap_file_chunks builds"""
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=30_000, seed_config=34)
    path = str(tmp_path / "16386")
    XF.write_heap_relation(tbl, path)
    want = XF.heap_file_chunks(tbl, path, pages_per_chunk=100)
    got = XF.heap_file_iovec(tbl, path, pages_per_chunk=100, io_pages=7)
    assert len(got) == len(want)
    raw = open(path, "rb").read()
    for g, w in zip(got, want):
        buf = np.zeros(g["length"], dtype=np.uint8)
        buf[:g["base_offset"]] = g["head"]
        npages = 0
        for m_off, fchunk, nr in g["iov"]:
            assert nr <= 7
            dst = g["base_offset"] + m_off
            buf[dst:dst + nr * XF.IO_PAGE] = np.frombuffer(
                raw[fchunk * XF.IO_PAGE:(fchunk + nr) * XF.IO_PAGE], dtype=np.uint8)
            npages += nr
        assert npages * XF.IO_PAGE == g["length"] - g["base_offset"]
        assert buf.tobytes() == w.tobytes()

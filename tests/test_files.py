"""Chunk producers over files (relscan.c / Arrow_Fdw counterparts): a heap
relation segment file read back into KDS_FORMAT_BLOCK chunks is the same
chunks, byte for byte, as the ones built in memory; an Arrow IPC file
with a dictionary-encoded text column becomes KDS_FORMAT_ARROW chunks the
oracle (and the device, test_gpu_files.py) group by that column; the
reference's own Arrow test file reads back as the CSV of its rows."""
import csv
import os
import sys

import numpy as np
import pytest

import xb_configs as C
import xb_files as XF
import xb_final as F
import xb_oracle as O
from xb_producer import Agg, Const, Func, SessionBuilder, Var, BoolOp

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import ref_fixtures as G  # noqa: E402


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


# ------------------------------------------------ the reference's Arrow fixture
# PG-Strom's regression suite imports test/data/python_generated_data.arrow
# next to the CSV of the same rows and checks that they hold the same data
# (test/sql/arrow_python_data.sql).  Here the Arrow file goes through the
# chunk producer into KDS_FORMAT_ARROW chunks and is read back, row by row, by
# the oracle and by the reference's own ExecLoadVarsOuterArrow
# (src/xpu_common.cu, host-compiled under oracle/_ref); both must give the
# CSV's values.  Skipped where the reference tree is not present.
PY_DATA_COLS = ["a_int32", "b_int64", "e_double", "f_string", "g_enum", "i_date"]


def _reference_test_data(name):
    """The reference tree's test/data/<name>, next to the src/ directory
    PGSTROM_SRC names or oracle/_ref was built from."""
    import ref_pin
    src = os.environ.get("PGSTROM_SRC") or ref_pin.source_dir()
    path = os.path.join(os.path.dirname(os.path.abspath(src)), "test", "data", name) if src else None
    if not path or not os.path.exists(path):
        pytest.skip(f"the reference's test/data/{name} is not present")
    return path


def _python_data_csv():
    rows = []
    with open(_reference_test_data("python_generated_data.csv"), newline="") as f:
        for r in csv.DictReader(f):
            day = (np.datetime64(r["i_date"]) - np.datetime64("1970-01-01")).astype(np.int64)
            rows.append((int(r["a_int32"]), int(r["b_int64"]), float(r["e_double"]),
                         r["f_string"].encode(), r["g_enum"].encode(), int(day)))
    return rows


def python_data_row_session():
    """GROUP BY every loaded column but b and e (a, f, g, date) -> count(*),
    min(b), max(b), min(e), max(e): one group per row of the file, so the
    groups are the rows, as the regression test's EXCEPT compares them."""
    va, vb, ve = Var(0, 1, "int4"), Var(0, 2, "int8"), Var(0, 3, "float8")
    vf, vg, vd = Var(0, 4, "text"), Var(0, 5, "text"), Var(0, 6, "date")
    return SessionBuilder(0, C.DEVTASK_PREAGG | C.DEVKIND_GPU).build(
        groupby_keys=[va, vf, vg, vd],
        aggs=[Agg("NROWS_ANY"), Agg("PMIN_INT64", vb), Agg("PMAX_INT64", vb),
              Agg("PMIN_FP64", ve), Agg("PMAX_FP64", ve)],
        ngroups_estimate=100.0)


def python_data_enum_session(lo_day):
    """WHERE i_date >= lo_day GROUP BY g_enum -> count(*), sum(a::int8),
    sum(e), min(e), max(e)."""
    va, ve, vg, vd = Var(0, 1, "int4"), Var(0, 3, "float8"), Var(0, 5, "text"), Var(0, 6, "date")
    return SessionBuilder(0, C.DEVTASK_PREAGG | C.DEVKIND_GPU).build(
        scan_quals=Func("date_ge", [vd, Const("date", lo_day - C.UNIX_TO_PG_DAYS)], "bool"),
        groupby_keys=[vg],
        aggs=[Agg("NROWS_ANY"), Agg("PSUM_INT", Func("int4_to_int8", [va], "int8")),
              Agg("PSUM_FP", ve), Agg("PMIN_FP64", ve), Agg("PMAX_FP64", ve)],
        ngroups_estimate=8.0)


def _groups_of(sess, chunks):
    o = O.Oracle(sess)
    for ch in chunks:
        o.exec(ch)
    got = F.decode_kds_final(o.final(), sess)
    st = o.stats()
    o.close()
    return got, st


def test_reference_arrow_fixture_rows():
    rows = _python_data_csv()
    chunks, tdef = XF.arrow_ipc_chunks(_reference_test_data("python_generated_data.arrow"), PY_DATA_COLS)
    assert [c.typ for c in tdef.columns] == ["int4", "int8", "float8", "text", "text", "date"]
    sess = python_data_row_session()
    want = {}
    for a, b, e, s, g, d in rows:
        key = (a, s, g, d - C.UNIX_TO_PG_DAYS)
        assert key not in want
        want[key] = [1, (1, b), (1, b), (1, e), (1, e)]
    got, st = _groups_of(sess, chunks)
    assert st["nitems_raw"] == st["nitems_in"] == len(rows)
    assert F.compare_groups(got, want, rtol=0.0) == []
    import ref_pin
    if ref_pin.available():
        res = ref_pin.run(sess, chunks)
        assert res["nitems_in"] == len(rows)
        assert F.compare_groups(G.decode_groups(res, sess), want, rtol=0.0) == []


def test_reference_arrow_fixture_groups():
    rows = _python_data_csv()
    chunks, _ = XF.arrow_ipc_chunks(_reference_test_data("python_generated_data.arrow"), PY_DATA_COLS)
    lo_day = 18628                                   # 2021-01-01
    sess = python_data_enum_session(lo_day)
    want = {}
    for a, b, e, s, g, d in rows:
        if d < lo_day:
            continue
        w = want.setdefault((g,), [0, 0, 0.0, np.inf, -np.inf])
        w[0] += 1
        w[1] += a
        w[2] += e
        w[3] = min(w[3], e)
        w[4] = max(w[4], e)
    want = {k: [n, (n, sa), (n, se), (1, mn), (1, mx)] for k, (n, sa, se, mn, mx) in want.items()}
    got, st = _groups_of(sess, chunks)
    assert st["nitems_in"] == sum(w[0] for w in want.values())
    assert F.compare_groups(got, want, rtol=0.0) == []
    import ref_pin
    if ref_pin.available():
        res = ref_pin.run(sess, chunks)
        assert res["nitems_in"] == st["nitems_in"]
        assert F.compare_groups(G.decode_groups(res, sess), want, rtol=0.0) == []


def test_arrow_int16_and_bool_columns(tmp_path):
    """Arrow Int16 keys and a bit-packed Bool filter with NULLs, in record
    batches of 7,001 rows (each batch's last bitmap byte partly used): the
    oracle against the arrays, and, where oracle/_ref is built, the
    reference's own readers (xpu_int2 / xpu_bool_datum_arrow_read) against
    the same groups."""
    chunks, sess, expect, meta = C.arrow_int2_bool(str(tmp_path))
    nin = meta["nitems_in"]
    assert meta["types"] == ["int2", "bool", "int4", "int8"]
    got, st = _groups_of(sess, chunks)
    assert st["nitems_in"] == nin
    assert F.compare_groups(got, expect, rtol=0.0) == []
    import ref_pin
    if ref_pin.available():
        res = ref_pin.run(sess, chunks)
        assert res["nitems_in"] == nin
        assert F.compare_groups(G.decode_groups(res, sess), expect, rtol=0.0) == []

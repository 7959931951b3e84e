"""The oracle against ground truth computed directly from the generator's
column arrays (no page or bytecode decoding on that side)."""
import xb_configs as C
import xb_final as F
import xb_oracle as O


def _want_c0(expect):
    return {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}


def _want_c1(expect):
    return {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}


def test_oracle_scan_groupby():
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=150_000)
    o = O.Oracle(sess)
    for ch in tbl.block_chunks(pages_per_chunk=300):
        o.exec(ch)
    st = o.stats()
    assert st["nitems_raw"] == meta["nitems_raw"] and st["nitems_in"] == meta["nitems_in"]
    assert F.compare_groups(F.decode_kds_final(o.final(), sess), _want_c0(expect)) == []
    o.close()


def test_oracle_join_groupby():
    fact, sess, km, expect, meta = C.join_groupby(nfact=200_000, ndim1=5000, ndim2=700)
    o = O.Oracle(sess, km)
    for ch in fact.block_chunks(pages_per_chunk=700):
        o.exec(ch)
    st = o.stats()
    assert st["nitems_out"] == meta["nitems_out"]
    assert st["depth_out"][:2] == meta["depth_out"]
    assert F.compare_groups(F.decode_kds_final(o.final(), sess), _want_c1(expect)) == []
    o.close()


def test_oracle_every_partial_state_form():
    # count, count(x), min/max int and float8, sum float8, avg numeric,
    # stddev and covar partial states against the column arrays
    tbl, sess, _, expect, meta = C.wide_groupby(nrows=60_000, ngroups=500)
    o = O.Oracle(sess)
    for ch in tbl.block_chunks(pages_per_chunk=100):
        o.exec(ch)
    assert o.stats()["nitems_in"] == meta["nitems_in"]
    assert F.compare_groups(F.decode_kds_final(o.final(), sess), expect) == []
    o.close()


def test_oracle_all_filtered_out():
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=5000, a_limit=0)
    o = O.Oracle(sess)
    for ch in tbl.block_chunks():
        o.exec(ch)
    assert expect == {}
    assert F.decode_kds_final(o.final(), sess) == {}
    o.close()


def _row_format(buf):
    import struct
    fmt = bytes(buf)[24:25]
    nslots = struct.unpack_from("<I", bytes(buf), 40)[0]
    return fmt, nslots


def test_oracle_no_group_by():
    # an aggregate without GROUP BY keys: one tuple in a KDS_FORMAT_ROW
    # kds_final with no hash slots; max(float8) is the maximum
    tbl, sess, _, expect, meta = C.scan_nogroup(nrows=120_000)
    o = O.Oracle(sess)
    for ch in tbl.block_chunks(pages_per_chunk=200):
        o.exec(ch)
    assert o.stats()["nitems_in"] == meta["nitems_in"]
    out = o.final()
    assert _row_format(out) == (b"r", 0)
    got = F.decode_kds_final(out, sess)
    assert list(got) == [()]
    assert F.compare_groups(got, expect) == []
    o.close()


def test_oracle_no_group_by_no_rows():
    # no qualifying row: no tuple (the reference creates the tuple only when
    # rows reach the aggregation, cuda_gpupreagg.cu:2246-2247)
    tbl, sess, _, expect, meta = C.scan_nogroup(nrows=5000, a_limit=0)
    o = O.Oracle(sess)
    for ch in tbl.block_chunks():
        o.exec(ch)
    assert expect == {}
    assert F.decode_kds_final(o.final(), sess) == {}
    o.close()


def test_oracle_arrow_nulls_and_short_buffers():
    # validity bitmaps on every column (NULL group keys form a group of their
    # own, NULL dates fail the filter, NULL arguments are skipped) and a v2
    # values buffer that ends before its chunk (those rows read as NULL)
    chunks, sess, expect, meta = C.arrow_nulls(nrows=80_000, nkeys=700, rows_per_chunk=30_000)
    o = O.Oracle(sess)
    for ch in chunks:
        o.exec(ch)
    got = F.decode_kds_final(o.final(), sess)
    st = o.stats()
    o.close()
    assert st["nitems_in"] == meta["nitems_in"]
    assert (None,) in got
    assert F.compare_groups(got, expect) == []


def test_oracle_skips_invalidated_line_pointers():
    """Pages whose line pointers are partly LP_UNUSED, LP_DEAD or
    LP_REDIRECT (as relscan.c leaves pages that are not all-visible, and as
    HOT pruning leaves them): only LP_NORMAL items are rows, as the
    reference's page walkers read them."""
    chunks, sess, expect, meta = C.scan_groupby_filtered(nrows=80_000, frac=0.2)
    assert meta["nitems_raw"] < 80_000 * 0.85
    o = O.Oracle(sess)
    for ch in chunks:
        o.exec(ch)
    st = o.stats()
    assert st["nitems_raw"] == meta["nitems_raw"] and st["nitems_in"] == meta["nitems_in"]
    assert F.compare_groups(F.decode_kds_final(o.final(), sess), _want_c0(expect)) == []
    o.close()


def test_oracle_row_chunks():
    """KDS_FORMAT_ROW outer chunks (kern_tupitems, row index from the
    chunk's end) of the same tables: the oracle's groups equal the arrays'
    and those of the heap chunks, with NULLs, 4-byte varlena headers and
    long numerics."""
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=50_000)
    o = O.Oracle(sess)
    for ch in tbl.row_chunks(rows_per_chunk=12_000):
        o.exec(ch)
    st = o.stats()
    assert st["nitems_raw"] == meta["nitems_raw"] and st["nitems_in"] == meta["nitems_in"]
    assert F.compare_groups(F.decode_kds_final(o.final(), sess), _want_c0(expect)) == []
    o.close()
    tbl, sess, _, _, _ = C.long_varlena_groupby(nrows=10_000)
    got = []
    for chunks in (tbl.row_chunks(rows_per_chunk=3_000), tbl.block_chunks(pages_per_chunk=50)):
        o = O.Oracle(sess)
        for ch in chunks:
            o.exec(ch)
        got.append(F.decode_kds_final(o.final(), sess))
        o.close()
    assert F.compare_groups(got[0], got[1], rtol=0.0) == []

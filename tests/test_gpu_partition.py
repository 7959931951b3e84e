"""Partitioned aggregation: a keyed GROUP BY into a global table several
times L2 defers every row's group update as a record bucketed by table
slot and replays the buckets in order (prepared batches by default,
XPU_B200_PARTITION=1 forces it, =0 disables it).  The groups must be those
of the in-place path: integer and numeric states exact, float states
within the float tolerance, on every partial-state form."""
import pytest

import xb_configs as C
import xb_final as F
import xpu_b200

pytestmark = pytest.mark.gpu


def _run(device, sess, chunks):
    s = xpu_b200.Session(device, sess)
    try:
        ups = [device.upload(c) for c in chunks]
        b = s.batch([p for _, p in ups])
        b.exec()
        b.close()
        final, res = s.final()
        info = s.info()
    finally:
        s.close()
        for base, _ in ups:
            device.free(base)
    return final, info


def test_partitioned_arrow_groupby(device, monkeypatch):
    monkeypatch.delenv("XPU_B200_PARTITION", raising=False)     # the default: on for this batch
    chunks, _, expect, meta = C.arrow_groupby(nrows=3_000_000, nkeys=1_000_000, rows_per_chunk=500_000,
                                              seed_config=81)
    # a 10M-group estimate: a 3.6 GB table, far beyond L2
    sess = C.arrow_groupby_session(ngroups_estimate=10_000_000.0)
    final, info = _run(device, sess, chunks)
    assert info["partition_used"] and info["partitions"] >= 8, info
    assert F.compare_groups(F.decode_kds_final(final, sess), expect) == []


def test_partitioned_every_state_form(device, monkeypatch):
    monkeypatch.setenv("XPU_B200_PARTITION", "1")
    tbl, _, _, expect, meta = C.wide_groupby(nrows=300_000, ngroups=3000, seed_config=82)
    sess = C.wide_groupby_session(ngroups=2_000_000)          # a table far larger than L2
    final, info = _run(device, sess, tbl.block_chunks(pages_per_chunk=256))
    assert info["partition_used"], info
    assert F.compare_groups(F.decode_kds_final(final, sess), expect) == []


def test_partitioned_arrow_nulls(device, monkeypatch):
    # NULL group keys and NULL arguments travel through the deferred
    # records' NULL masks and the replay
    monkeypatch.delenv("XPU_B200_PARTITION", raising=False)
    chunks, _, expect, meta = C.arrow_nulls(nrows=600_000, nkeys=200_000, rows_per_chunk=200_000, seed_config=84)
    sess = C.arrow_groupby_session(ngroups_estimate=10_000_000.0)
    final, info = _run(device, sess, chunks)
    assert info["partition_used"], info
    got = F.decode_kds_final(final, sess)
    assert (None,) in got
    assert F.compare_groups(got, expect) == []


def test_in_place_without_the_switch(device, monkeypatch):
    monkeypatch.setenv("XPU_B200_PARTITION", "0")
    chunks, sess, expect, meta = C.arrow_groupby(nrows=1_000_000, nkeys=300_000, rows_per_chunk=500_000,
                                                 seed_config=83)
    final, info = _run(device, sess, chunks)
    assert not info["partition_used"]
    assert F.compare_groups(F.decode_kds_final(final, sess), expect) == []


def test_partitioned_text_keys(device, monkeypatch):
    # GROUP BY a text column (the record carries the key's length) with a
    # large estimate, against the oracle
    import xb_oracle as O
    from xb_producer import Agg, SessionBuilder, Var
    monkeypatch.setenv("XPU_B200_PARTITION", "1")
    fact, _, km, _, meta = C.join_groupby(nfact=1000, ndim1=200_000, ndim2=70, seed_config=84)
    dim1 = meta["dims"]["dim1"]
    sess = SessionBuilder(0, C.DEVTASK_PREAGG | C.DEVKIND_GPU).build(
        groupby_keys=[Var(0, 2, "text")], aggs=[Agg("NROWS_ANY"), Agg("PSUM_INT", Var(0, 1, "int4"))],
        ngroups_estimate=2_000_000.0)
    chunks = dim1.block_chunks(pages_per_chunk=256)
    final, info = _run(device, sess, chunks)
    assert info["partition_used"], info
    o = O.Oracle(sess)
    for ch in chunks:
        o.exec(ch)
    want = F.decode_kds_final(o.final(), sess)
    o.close()
    assert F.compare_groups(F.decode_kds_final(final, sess), want) == []


@pytest.mark.parametrize("cap", ["1", "700"])
def test_full_buckets_update_in_place(device, monkeypatch, cap):
    # buckets clipped to a few records: most rows of a group are updated in
    # place while others of the same group are deferred and replayed
    monkeypatch.setenv("XPU_B200_PARTITION", "1")
    monkeypatch.setenv("XPU_B200_PART_CAP", cap)
    tbl, _, _, expect, meta = C.wide_groupby(nrows=300_000, ngroups=3000, seed_config=85)
    sess = C.wide_groupby_session(ngroups=2_000_000)
    final, info = _run(device, sess, tbl.block_chunks(pages_per_chunk=256))
    assert info["partition_used"], info
    assert F.compare_groups(F.decode_kds_final(final, sess), expect) == []


def test_full_buckets_text_keys(device, monkeypatch):
    import xb_oracle as O
    from xb_producer import Agg, SessionBuilder, Var
    monkeypatch.setenv("XPU_B200_PARTITION", "1")
    monkeypatch.setenv("XPU_B200_PART_CAP", "300")
    fact, _, km, _, meta = C.join_groupby(nfact=1000, ndim1=200_000, ndim2=70, seed_config=86)
    dim1 = meta["dims"]["dim1"]
    sess = SessionBuilder(0, C.DEVTASK_PREAGG | C.DEVKIND_GPU).build(
        groupby_keys=[Var(0, 2, "text")], aggs=[Agg("NROWS_ANY"), Agg("PSUM_INT", Var(0, 1, "int4"))],
        ngroups_estimate=2_000_000.0)
    chunks = dim1.block_chunks(pages_per_chunk=256)
    final, info = _run(device, sess, chunks)
    assert info["partition_used"], info
    o = O.Oracle(sess)
    for ch in chunks:
        o.exec(ch)
    want = F.decode_kds_final(o.final(), sess)
    o.close()
    assert F.compare_groups(F.decode_kds_final(final, sess), want) == []


def test_staged_pages_do_not_defer_text_keys(device, monkeypatch):
    # with heap pages staged in shared memory the text key registers point
    # into the staging buffer, so partitioned aggregation stays off and the
    # groups are updated in place
    import xb_oracle as O
    from xb_producer import Agg, SessionBuilder, Var
    monkeypatch.setenv("XPU_B200_PARTITION", "1")
    monkeypatch.setenv("XPU_B200_JIT_STAGE", "1")
    fact, _, km, _, meta = C.join_groupby(nfact=1000, ndim1=200_000, ndim2=70, seed_config=87)
    dim1 = meta["dims"]["dim1"]
    sess = SessionBuilder(0, C.DEVTASK_PREAGG | C.DEVKIND_GPU).build(
        groupby_keys=[Var(0, 2, "text")], aggs=[Agg("NROWS_ANY"), Agg("PSUM_INT", Var(0, 1, "int4"))],
        ngroups_estimate=2_000_000.0)
    chunks = dim1.block_chunks(pages_per_chunk=256)
    final, info = _run(device, sess, chunks)
    assert not info["partition_used"], info
    o = O.Oracle(sess)
    for ch in chunks:
        o.exec(ch)
    want = F.decode_kds_final(o.final(), sess)
    o.close()
    assert F.compare_groups(F.decode_kds_final(final, sess), want) == []

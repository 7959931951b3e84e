"""Group tables that outgrow their estimate: the table grows and the work
resumes, as the reference's service expands kds_final and resumes the
suspended kernel on SUSPEND_NO_SPACE (gpu_service.c:2418-2470, :3872-3879;
cuda_gpujoin.cu:1098-1103).  One session, an estimate far too low, and the
exact result: every row applied once (statistics exact), integer and
numeric states bit-exact, float sums within 1e-12 of the row-ordered sum
(of the sum of magnitudes where terms cancel).  Both kernels; single-chunk
ExecTask, prepared batches, partitioned aggregation, text keys whose arena
grows, shared-table merges, and MergeFinal."""
import numpy as np
import pytest

import xb_configs as C
import xb_final as F
import xb_oracle as O
import xpu_b200

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["jit", "vm"])
def kernel(request, monkeypatch):
    monkeypatch.setenv("XPU_B200_JIT", "1" if request.param == "jit" else "0")
    return request.param


def _run(device, sess, chunks, batch=False, kmrels=None, nrels=0):
    s = xpu_b200.Session(device, sess, kmrels, nrels)
    ups = []
    tot = {"nitems_raw": 0, "nitems_in": 0, "nitems_out": 0}
    try:
        if batch:
            ups = [device.upload(c) for c in chunks]
            b = s.batch([p for _, p in ups])
            r = b.exec()
            b.close()
            for k in tot:
                tot[k] += r[k]
        else:
            for ch in chunks:
                r = s.exec(ch)
                for k in tot:
                    tot[k] += r[k]
        info = s.info()
        final, res = s.final()
    finally:
        s.close()
        for base, _ in ups:
            device.free(base)
    return final, tot, info, res


def _c0_truth(expect):
    return {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}


@pytest.mark.parametrize("batch", [False, True])
def test_estimate_one_sixty_thousand_groups(device, kernel, batch):
    # 60,000 groups into a session sized for one (a 2,048-slot table)
    tbl, _, _, expect, meta = C.scan_groupby(nrows=200_000, ngroups=60_000, a_limit=1000, seed_config=72)
    sess = C.scan_groupby_session(a_limit=1000, ngroups=1)
    chunks = tbl.block_chunks(pages_per_chunk=256)
    final, tot, info, res = _run(device, sess, chunks, batch=batch)
    assert info["gtable_grew"] >= 1, info
    assert tot["nitems_raw"] == meta["nitems_raw"] and tot["nitems_in"] == meta["nitems_in"]
    assert tot["nitems_out"] == meta["nitems_out"]
    got = F.decode_kds_final(final, sess)
    assert F.compare_groups(got, _c0_truth(expect)) == []
    assert res["final_nitems"] == len(expect)


def test_arrow_estimate_hundred_times_too_low(device, kernel):
    # the Arrow group-by shape with 1M keys and an estimate of 10,000
    chunks, _, expect, meta = C.arrow_groupby(nrows=2_000_000, nkeys=1_000_000, rows_per_chunk=500_000,
                                              seed_config=73)
    sess = C.arrow_groupby_session(ngroups_estimate=10_000.0)
    final, tot, info, res = _run(device, sess, chunks, batch=True)
    assert info["gtable_grew"] >= 2, info
    assert tot["nitems_raw"] == meta["nitems_raw"] and tot["nitems_in"] == meta["nitems_in"]
    assert F.compare_groups(F.decode_kds_final(final, sess), expect) == []


def test_partitioned_replay_finds_the_table_full(device, monkeypatch):
    # partitioned aggregation forced over a 1M-slot table (117 MB) while
    # 1.25M groups arrive in one launch: the replay, which cannot stop,
    # leaves the records the full table has no room for until it grew
    monkeypatch.setenv("XPU_B200_JIT", "1")
    monkeypatch.setenv("XPU_B200_PARTITION", "1")
    chunks, _, expect, meta = C.arrow_groupby(nrows=8_000_000, nkeys=3_000_000, rows_per_chunk=1_000_000,
                                              seed_config=74)
    sess = C.arrow_groupby_session(ngroups_estimate=150_000.0)
    final, tot, info, res = _run(device, sess, chunks, batch=True)
    assert info["partition_used"] and info["gtable_grew"] >= 1, info
    assert tot["nitems_in"] == meta["nitems_in"]
    assert F.compare_groups(F.decode_kds_final(final, sess), expect) == []


def test_text_keys_and_the_key_arena_grow(device, kernel):
    # 150,000 distinct text keys of up to 300 bytes into a session sized for
    # 100 groups: the table and the key arena both grow, key pointers move
    tbl, _, _, expect, meta = C.long_varlena_groupby(nrows=300_000, ngroups=150_000, seed_config=75)
    sess = C.long_varlena_session(ngroups=100)
    chunks = tbl.block_chunks(pages_per_chunk=512)
    final, tot, info, res = _run(device, sess, chunks)
    assert info["gtable_grew"] >= 1, info
    assert tot["nitems_in"] == meta["nitems_in"]
    assert F.compare_groups(F.decode_kds_final(final, sess), expect, rtol=0.0) == []


def test_join_group_keys_beyond_the_estimate(device, kernel):
    # GROUP BY an inner text column with 3,000 distinct values in a session
    # estimated at 25 groups: shared-table merges find the table full
    fact, sess, km, expect, meta = C.join_groupby(nfact=400_000, ndim1=20_000, ndim2=2_000,
                                                  regions=C.long_strings(3000, lo=8, hi=60), seed_config=76)
    chunks = fact.block_chunks(pages_per_chunk=300)
    final, tot, info, res = _run(device, sess, chunks, kmrels=km, nrels=2)
    assert info["gtable_grew"] >= 1, info
    assert tot["nitems_out"] == meta["nitems_out"]
    truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    assert F.compare_groups(F.decode_kds_final(final, sess), truth, rtol=0.0) == []


def test_merge_final_grows_the_table(device):
    # a 200,000-group kds_final merged into a session estimated at one group
    chunks, sess, expect, meta = C.arrow_groupby(nrows=600_000, nkeys=200_000, rows_per_chunk=300_000,
                                                 seed_config=77)
    final, _, _, _ = _run(device, sess, chunks)
    small = C.arrow_groupby_session(ngroups_estimate=1.0)
    s = xpu_b200.Session(device, small)
    try:
        s.merge_final(final)
        info = s.info()
        merged, res = s.final()
    finally:
        s.close()
    assert info["gtable_grew"] >= 1, info
    assert F.compare_groups(F.decode_kds_final(merged, small), expect) == []


def test_growth_matches_the_oracle_every_state_form(device, kernel):
    # every partial-state form through a growth: equal to the oracle
    tbl, _, _, expect, meta = C.wide_groupby(nrows=300_000, ngroups=40_000, seed_config=78)
    sess = C.wide_groupby_session(ngroups=10)
    chunks = tbl.block_chunks(pages_per_chunk=256)
    final, tot, info, res = _run(device, sess, chunks, batch=True)
    assert info["gtable_grew"] >= 1, info
    got = F.decode_kds_final(final, sess)
    assert F.compare_groups(got, expect) == []
    o = O.Oracle(sess)
    for ch in chunks:
        o.exec(ch)
    want = F.decode_kds_final(o.final(), sess)
    o.close()
    for k in want:
        assert got[k][:4] == want[k][:4] and got[k][7] == want[k][7], k

"""The error and suspend protocol on the GPU (kern_errorbuf codes): an
expression error in a row stops the chunk with the reference's message,
as the oracle does; a group table that cannot grow within the device's
memory budget returns ERRCODE_SUSPEND_NO_SPACE instead of losing groups;
and a session stays usable for the caller to close after either.  Both
kernels.  (A table that can grow does: tests/test_gpu_growth.py.)"""
import pytest

import xb_configs as C
import xb_oracle as O
import xpu_b200

pytestmark = pytest.mark.gpu


@pytest.fixture(params=["jit", "vm"])
def kernel(request, monkeypatch):
    monkeypatch.setenv("XPU_B200_JIT", "1" if request.param == "jit" else "0")
    return request.param


def test_int8_overflow_in_join_expression(device, kernel):
    # qty * price with price up to 4e17 and qty up to 50 leaves int8
    fact, sess, km, _, _ = C.join_groupby(nfact=50_000, ndim1=2000, ndim2=300, seed_config=71,
                                          price_hi=400_000_000_000_000_000)
    chunks = fact.block_chunks(pages_per_chunk=64)
    o = O.Oracle(sess, km)
    with pytest.raises(Exception, match="out of range"):
        for ch in chunks:
            o.exec(ch)
    o.close()
    s = xpu_b200.Session(device, sess, km, 2)
    try:
        with pytest.raises(xpu_b200.XpuB200Error, match="integer value out of range"):
            for ch in chunks:
                s.exec(ch)
    finally:
        s.close()


def test_group_table_that_cannot_grow_suspends(kernel):
    # 60,000 groups into a session sized for one, on a device whose memory
    # budget caps the group table at 65,536 slots: the table grows as far
    # as the budget allows, then SUSPEND_NO_SPACE is returned instead of
    # losing groups, and the session can still be closed
    tbl, _, _, _, _ = C.scan_groupby(nrows=200_000, ngroups=60_000, a_limit=1000, seed_config=72)
    dev = xpu_b200.Device(0, hbm_budget=24 << 20)
    try:
        s = xpu_b200.Session(dev, C.scan_groupby_session(a_limit=1000, ngroups=1))
        try:
            with pytest.raises(xpu_b200.XpuB200Error) as ei:
                for ch in tbl.block_chunks(pages_per_chunk=256):
                    s.exec(ch)
            assert ei.value.errcode == ord("d") or "no space" in str(ei.value), str(ei.value)
        finally:
            s.close()
    finally:
        dev.close()


@pytest.mark.parametrize("estimate", [64, 100_000])
def test_bounded_wait_on_a_busy_entry_times_out(kernel, monkeypatch, estimate):
    # every global group entry is left BUSY, as if its creator never
    # published it, and the wait on such an entry is cut to 10,000 spins:
    # the launch stops with the wait-timeout error (through the CTA's merge
    # of its shared table when there is one, estimate 64, or on the rows'
    # own lookups, estimate 100,000), promptly, the session closes, and the
    # device runs the next session correctly
    import time
    import xb_final as F
    monkeypatch.setenv("XPU_B200_WAIT_LIMIT", "10000")
    monkeypatch.setenv("XPU_B200_TEST_BUSY_GROUPS", "1")
    tbl, _, _, expect, meta = C.scan_groupby(nrows=60_000, seed_config=73)
    chunks = tbl.block_chunks(pages_per_chunk=64)
    dev = xpu_b200.Device(0)
    try:
        s = xpu_b200.Session(dev, C.scan_groupby_session(ngroups=estimate))
        t0 = time.perf_counter()
        try:
            with pytest.raises(xpu_b200.XpuB200Error, match="wait timed out"):
                for ch in chunks:
                    s.exec(ch)
        finally:
            s.close()
        assert time.perf_counter() - t0 < 20.0
        monkeypatch.delenv("XPU_B200_TEST_BUSY_GROUPS")
        s2 = xpu_b200.Session(dev, C.scan_groupby_session(ngroups=estimate))
        try:
            for ch in chunks:
                s2.exec(ch)
            final, _ = s2.final()
        finally:
            s2.close()
        truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
        assert F.compare_groups(F.decode_kds_final(final, C.scan_groupby_session(ngroups=estimate)), truth) == []
    finally:
        dev.close()

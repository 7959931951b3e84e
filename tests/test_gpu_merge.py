"""Merge of partial-aggregation results (xpuB200MergeFinal), as between the
GPUs of a multi-GPU GpuPreAgg: a table's chunks are split between sessions
and the other sessions' kds_final buffers are merged into the first
session's group table.  Its kds_final must then hold every group with the
states one session over all chunks would have: integer and numeric states
exact, float8 sums within 1e-12 of their terms' magnitude."""
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


def _split_run(device, sess, chunks, nparts, km=None, nrels=0, on_device=False):
    """chunk i runs on session i % nparts; the other sessions' kds_final is
    merged into session 0's; returns session 0's kds_final"""
    parts = [xpu_b200.Session(device, sess, km, nrels) for _ in range(nparts)]
    bases = []
    try:
        for i, ch in enumerate(chunks):
            parts[i % nparts].exec(ch)
        for s in parts[1:]:
            f, _ = s.final()
            if f is None:
                continue
            if on_device:
                base, p = device.upload(f, align_pages=False)
                bases.append(base)
                parts[0].merge_final(p, on_device=True)
            else:
                parts[0].merge_final(f)
        final, res = parts[0].final()
        return final, res
    finally:
        for s in parts:
            s.close()
        for b in bases:
            device.free(b)


@pytest.mark.parametrize("on_device", [False, True])
def test_merge_scan_groupby(device, kernel, on_device):
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=200_000, ngroups=5000)
    chunks = tbl.block_chunks(pages_per_chunk=64)
    final, res = _split_run(device, sess, chunks, 2, on_device=on_device)
    truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
    assert F.compare_groups(F.decode_kds_final(final, sess), truth) == []
    assert res["final_nitems"] == len(truth)


def test_merge_every_partial_state_form(device, kernel):
    tbl, sess, _, expect, meta = C.wide_groupby(nrows=200_000, ngroups=3000)
    chunks = tbl.block_chunks(pages_per_chunk=64)
    final, _ = _split_run(device, sess, chunks, 3)
    got = F.decode_kds_final(final, sess)
    assert F.compare_groups(got, expect) == []
    o = O.Oracle(sess)
    for ch in chunks:
        o.exec(ch)
    want = F.decode_kds_final(o.final(), sess)
    o.close()
    assert set(got) == set(want)


def test_merge_join_groupby_text_keys(device):
    fact, sess, km, expect, meta = C.join_groupby(nfact=300_000, ndim1=5_000, ndim2=700)
    chunks = fact.block_chunks(pages_per_chunk=100)
    final, _ = _split_run(device, sess, chunks, 4, km=km, nrels=2)
    truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    assert F.compare_groups(F.decode_kds_final(final, sess), truth) == []


def test_merge_arrow_groupby_many_groups(device):
    chunks, sess, expect, meta = C.arrow_groupby(nrows=600_000, nkeys=200_000, rows_per_chunk=100_000)
    final, res = _split_run(device, sess, chunks, 2)
    assert F.compare_groups(F.decode_kds_final(final, sess), expect) == []
    assert res["final_nitems"] == len(expect)


def test_merge_into_session_without_chunks(device):
    tbl, sess, _, expect, meta = C.wide_groupby(nrows=50_000, ngroups=400)
    a = xpu_b200.Session(device, sess)
    b = xpu_b200.Session(device, sess)
    try:
        for ch in tbl.block_chunks(pages_per_chunk=100):
            b.exec(ch)
        fb, _ = b.final()
        a.merge_final(fb)
        fa, _ = a.final()
        assert F.compare_groups(F.decode_kds_final(fa, sess), expect) == []
        assert F.decode_kds_final(fa, sess) == F.decode_kds_final(fb, sess)
    finally:
        a.close()
        b.close()


def test_merge_rejects_another_sessions_layout(device):
    tbl, ssess, _, _, _ = C.scan_groupby(nrows=20_000)
    fact, jsess, km, _, _ = C.join_groupby(nfact=20_000, ndim1=500, ndim2=70)
    s = xpu_b200.Session(device, ssess)
    j = xpu_b200.Session(device, jsess, km, 2)
    try:
        for ch in fact.block_chunks():
            j.exec(ch)
        fj, _ = j.final()
        with pytest.raises(xpu_b200.XpuB200Error, match="not this session"):
            s.merge_final(fj)
    finally:
        s.close()
        j.close()

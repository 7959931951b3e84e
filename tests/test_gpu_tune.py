"""Launch-shape autotuning (xpuB200BatchTune): every measured shape is a
valid kernel, the session keeps the fastest, later sessions of the same
plan shape adopt it, and the results are the same as untuned."""
import pytest

import xb_configs as C
import xb_final as F
import xpu_b200

pytestmark = pytest.mark.gpu


def _upload(device, chunks):
    ups = [device.upload(c) for c in chunks]
    return [b for b, _ in ups], [p for _, p in ups]


def test_tune_join_groupby_and_adopt(device):
    fact, sess, km, expect, meta = C.join_groupby(nfact=1_000_000, ndim1=200_000, ndim2=10_000, seed_config=21)
    chunks = fact.block_chunks(pages_per_chunk=2048)
    bases, ptrs = _upload(device, chunks)
    truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    s = xpu_b200.Session(device, sess, km, 2)
    s2 = xpu_b200.Session(device, sess, km, 2)
    try:
        b = s.batch(ptrs)
        rep = b.tune()
        shapes = [(c["ctas_per_sm"], c["sm_groups"]) for c in rep["candidates"]]
        assert [m for m, _ in shapes][:5] == [2, 3, 4, 6, 8], rep
        assert all(c["kernel"] == "jit" and c["ms"] > 0 for c in rep["candidates"]), rep
        best = rep["best"]
        assert best["ms"] == min(c["ms"] for c in rep["candidates"])
        r = b.exec()
        assert r["nitems_out"] == meta["nitems_out"]
        info = s.info()
        assert info["jit_ctas_per_sm"] == best["ctas_per_sm"] and info["sm_cap"] == best["sm_groups"]
        final, _ = s.final()
        assert F.compare_groups(F.decode_kds_final(final, sess), truth) == []
        b.close()
        # another session of the same plan shape adopts the tuned shape
        for p in ptrs:
            s2.exec(p, on_device=True)
        info2 = s2.info()
        assert info2["jit_ctas_per_sm"] == best["ctas_per_sm"] and info2["sm_cap"] == best["sm_groups"]
        f2, _ = s2.final()
        assert F.compare_groups(F.decode_kds_final(f2, sess), truth) == []
    finally:
        s.close()
        s2.close()
        for x in bases:
            device.free(x)


@pytest.mark.parametrize("jit", ["1", "0"])
def test_tune_shared_table_sizes(device, monkeypatch, jit):
    monkeypatch.setenv("XPU_B200_JIT", jit)
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=400_000, seed_config=22)
    chunks = tbl.block_chunks(pages_per_chunk=1000)
    bases, ptrs = _upload(device, chunks)
    truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
    s = xpu_b200.Session(device, sess)
    try:
        b = s.batch(ptrs)
        rep = b.tune()
        sm0 = rep["default_sm_groups"]
        assert sm0 > 0
        sms = {c["sm_groups"] for c in rep["candidates"]}
        assert {sm0, 0} <= sms, rep
        kinds = {c["kernel"] for c in rep["candidates"]}
        assert kinds == ({"jit"} if jit == "1" else {"vm"}), rep
        r = b.exec()
        assert r["nitems_in"] == meta["nitems_in"]
        final, _ = s.final()
        assert F.compare_groups(F.decode_kds_final(final, sess), truth) == []
        b.close()
    finally:
        s.close()
        for x in bases:
            device.free(x)


def test_tune_after_exec_is_rejected(device):
    tbl, sess, _, _, _ = C.scan_groupby(nrows=50_000, seed_config=23)
    chunks = tbl.block_chunks(pages_per_chunk=400)
    bases, ptrs = _upload(device, chunks)
    s = xpu_b200.Session(device, sess)
    try:
        s.exec(ptrs[0], on_device=True)
        b = s.batch(ptrs)
        with pytest.raises(xpu_b200.XpuB200Error, match="before it executes"):
            b.tune()
        b.close()
    finally:
        s.close()
        for x in bases:
            device.free(x)

"""Parity of the CUDA path (through the C ABI) with the CPU oracle and with
the generator's ground truth.  Integer / numeric / text states bit-exact;
float8 sums within 1e-12 relative of the FP64 row-ordered sum.

Every test runs twice: on the session-specialised kernel ("jit", built by
NVRTC at the first launch) and on the interpreting kernel ("vm",
XPU_B200_JIT=0); each run checks that the intended kernel executed."""
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


def check_kernel(s, kernel):
    info = s.info()
    ran = set(info["kernels"].values())
    assert ran == {kernel}, f"expected the {kernel} kernel, ran {info['kernels']}: {info['jit_msg']}"


def run_gpu(device, sess, chunks, kmrels=None, nrels=0, on_device=False, kernel=None):
    s = xpu_b200.Session(device, sess, kmrels, nrels)
    totals = {"nitems_raw": 0, "nitems_in": 0, "nitems_out": 0, "depth_out": [0] * nrels}
    bufs = []
    for ch in chunks:
        if on_device:
            base, p = device.upload(ch)
            bufs.append(base)
            r = s.exec(p, on_device=True)
        else:
            r = s.exec(ch)
        for k in ("nitems_raw", "nitems_in", "nitems_out"):
            totals[k] += r[k]
        for d in range(nrels):
            totals["depth_out"][d] += r["depth_out"][d]
    if kernel:
        check_kernel(s, kernel)
    final, res = s.final()
    s.close()
    for b in bufs:
        device.free(b)
    return final, totals, res


def run_oracle(sess, chunks, kmrels=None):
    o = O.Oracle(sess, kmrels)
    for ch in chunks:
        o.exec(ch)
    out = o.final()
    st = o.stats()
    o.close()
    return out, st


@pytest.mark.parametrize("nrows,ppc", [(20_000, 64), (400_000, 1000)])
def test_scan_groupby_parity(device, kernel, nrows, ppc):
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=nrows)
    chunks = tbl.block_chunks(pages_per_chunk=ppc)
    final, st, res = run_gpu(device, sess, chunks, kernel=kernel)
    assert st["nitems_raw"] == meta["nitems_raw"]
    assert st["nitems_in"] == meta["nitems_in"]
    got = F.decode_kds_final(final, sess)
    ofinal, ost = run_oracle(sess, chunks)
    want = F.decode_kds_final(ofinal, sess)
    assert F.compare_groups(got, want) == []
    truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
    assert F.compare_groups(got, truth) == []
    assert res["final_nitems"] == len(truth)


def test_every_partial_state_form_parity(device, kernel):
    # count(x), min/max of int4 / int8 / float8, sum float8, avg numeric,
    # stddev and covar states, against the column arrays and the oracle
    tbl, sess, _, expect, meta = C.wide_groupby(nrows=300_000, ngroups=3000)
    chunks = tbl.block_chunks(pages_per_chunk=256)
    final, st, res = run_gpu(device, sess, chunks, kernel=kernel)
    assert st["nitems_in"] == meta["nitems_in"]
    got = F.decode_kds_final(final, sess)
    assert F.compare_groups(got, expect) == []
    ofinal, _ = run_oracle(sess, chunks)
    want = F.decode_kds_final(ofinal, sess)
    assert set(got) == set(want)
    for k in want:
        # integer and numeric states bit-exact with the oracle
        assert got[k][:4] == want[k][:4] and got[k][7] == want[k][7], k


def test_min_max_stddev_in_shared_tables(device, kernel):
    """min / max of int4, int8 and float8 and stddev with a group estimate
    small enough for the per-CTA shared-memory group table (on the
    specialised kernel its own state form, updated with shared-memory
    atomics and merged into the global table at CTA exit): equal to the
    oracle."""
    from xb_producer import Agg, Const, Func, SessionBuilder, Var
    va, vb, vg = Var(0, 2, "int4"), Var(0, 3, "float8"), Var(0, 5, "int4")
    sess = SessionBuilder(0, C.DEVTASK_PREAGG | C.DEVKIND_GPU).build(
        scan_quals=Func("int4lt", [va, Const("int4", 800)], "bool"),
        groupby_keys=[vg],
        aggs=[Agg("NROWS_ANY"), Agg("PMIN_INT32", va), Agg("PMAX_INT64", Func("int4_to_int8", [va], "int8")),
              Agg("PMIN_FP64", vb), Agg("PMAX_FP64", vb), Agg("STDDEV", vb)],
        ngroups_estimate=200.0)
    tbl, _, _, _, _ = C.scan_groupby(nrows=300_000, ngroups=200, seed_config=9)
    chunks = tbl.block_chunks(pages_per_chunk=256)
    s = xpu_b200.Session(device, sess)
    try:
        assert s.info()["sm_cap"] > 0, s.info()
        for ch in chunks:
            s.exec(ch)
        check_kernel(s, kernel)
        final, _ = s.final()
    finally:
        s.close()
    got = F.decode_kds_final(final, sess)
    ofinal, _ = run_oracle(sess, chunks)
    want = F.decode_kds_final(ofinal, sess)
    assert len(want) == 200 and set(got) == set(want)
    for k in want:
        assert got[k][:5] == want[k][:5], k          # counts, min and max exact
    # the stddev state (n, sum, sum of squares) against the column arrays
    a, b, bnull, g = (tbl.col("a").values, tbl.col("b").values, tbl.col("b").nulls, tbl.col("g").values)
    m = (a < 800) & ~bnull
    truth = {}
    for k in range(200):
        x = b[m & (g == k)]
        truth[(k,)] = [(len(x), F.Approx(float(np.sum(x)), float(np.abs(x).sum())),
                        F.Approx(float(np.sum(x * x)), float(np.sum(x * x))))]
    assert F.compare_groups({k: [v[5]] for k, v in got.items()}, truth) == []


def test_scan_groupby_device_resident(device, kernel):
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=100_000)
    chunks = tbl.block_chunks(pages_per_chunk=200)
    final, st, _ = run_gpu(device, sess, chunks, on_device=True, kernel=kernel)
    truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
    assert F.compare_groups(F.decode_kds_final(final, sess), truth) == []


def test_scan_groupby_empty_result(device, kernel):
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=10_000, a_limit=0)
    final, st, res = run_gpu(device, sess, tbl.block_chunks(), kernel=kernel)
    assert st["nitems_in"] == 0
    assert F.decode_kds_final(final, sess) == {}


@pytest.mark.parametrize("nfact,nd1,nd2,ppc", [(50_000, 2000, 300, 128), (1_000_000, 200_000, 10_000, 2048)])
def test_join_groupby_parity(device, kernel, nfact, nd1, nd2, ppc):
    fact, sess, km, expect, meta = C.join_groupby(nfact=nfact, ndim1=nd1, ndim2=nd2)
    chunks = fact.block_chunks(pages_per_chunk=ppc)
    final, st, res = run_gpu(device, sess, chunks, km, nrels=2, kernel=kernel)
    assert st["nitems_raw"] == meta["nitems_raw"]
    assert st["nitems_out"] == meta["nitems_out"]
    assert st["depth_out"] == meta["depth_out"]
    got = F.decode_kds_final(final, sess)
    truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    assert F.compare_groups(got, truth) == []
    ofinal, ost = run_oracle(sess, chunks, km)
    assert F.compare_groups(got, F.decode_kds_final(ofinal, sess)) == []


@pytest.mark.parametrize("stride,copies,miss", [(7, 1, 0.0), (1, 3, 0.2), (13, 2, 0.1)])
def test_join_probe_variants_parity(device, kernel, stride, copies, miss):
    """Sparse keys (hashed probe instead of direct addressing), repeated
    inner keys (several matches per probe) and fact rows without a match."""
    fact, sess, km, expect, meta = C.join_groupby(nfact=200_000, ndim1=5_000, ndim2=700, key_stride=stride,
                                                  dim1_copies=copies, miss_frac=miss)
    chunks = fact.block_chunks(pages_per_chunk=300)
    final, st, res = run_gpu(device, sess, chunks, km, nrels=2, kernel=kernel)
    assert st["nitems_out"] == meta["nitems_out"]
    assert st["depth_out"] == meta["depth_out"]
    got = F.decode_kds_final(final, sess)
    truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    assert F.compare_groups(got, truth) == []
    ofinal, _ = run_oracle(sess, chunks, km)
    assert F.compare_groups(got, F.decode_kds_final(ofinal, sess)) == []


@pytest.mark.parametrize("nrows,nkeys,rpc", [(300_000, 20_000, 100_000), (2_000_000, 1_000_000, 700_000)])
def test_arrow_groupby_parity(device, kernel, nrows, nkeys, rpc):
    chunks, sess, expect, meta = C.arrow_groupby(nrows=nrows, nkeys=nkeys, rows_per_chunk=rpc)
    final, st, res = run_gpu(device, sess, chunks, kernel=kernel)
    assert st["nitems_raw"] == meta["nitems_raw"]
    assert st["nitems_in"] == meta["nitems_in"]
    got = F.decode_kds_final(final, sess)
    assert F.compare_groups(got, expect) == []


@pytest.mark.parametrize("short_rows", [0, 100])
def test_arrow_nulls_parity(device, kernel, short_rows):
    """Arrow columns with validity bitmaps (NULL group keys, NULL dates in
    the filter, NULL arguments) and, with short_rows, a values buffer that
    ends before its chunk (those rows read as NULL): the groups of the
    oracle and of the arrays, on both kernels."""
    chunks, sess, expect, meta = C.arrow_nulls(nrows=300_000, nkeys=3_000, rows_per_chunk=100_000,
                                               short_rows=short_rows)
    final, st, res = run_gpu(device, sess, chunks, kernel=kernel)
    assert st["nitems_raw"] == meta["nitems_raw"]
    assert st["nitems_in"] == meta["nitems_in"]
    got = F.decode_kds_final(final, sess)
    assert (None,) in got
    assert F.compare_groups(got, expect) == []
    ofinal, _ = run_oracle(sess, chunks)
    assert F.compare_groups(got, F.decode_kds_final(ofinal, sess)) == []


def test_batch_matches_single_chunk_path(device, kernel):
    fact, sess, km, expect, meta = C.join_groupby(nfact=300_000, ndim1=20_000, ndim2=2_000)
    chunks = fact.block_chunks(pages_per_chunk=300)
    s = xpu_b200.Session(device, sess, km, 2)
    ups = [device.upload(c) for c in chunks]
    b = s.batch([p for _, p in ups])
    r = b.exec()
    check_kernel(s, kernel)
    assert r["nitems_raw"] == meta["nitems_raw"] and r["nitems_out"] == meta["nitems_out"]
    assert r["depth_out"] == meta["depth_out"]
    final, _ = s.final()
    b.close()
    s.close()
    for base, _ in ups:
        device.free(base)
    truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    assert F.compare_groups(F.decode_kds_final(final, sess), truth) == []


@pytest.mark.parametrize("nrows,ppc", [(30_000, 40), (600_000, 1500)])
def test_no_group_by_parity(device, kernel, nrows, ppc):
    """count(*), count(b), sum(a), sum(c), avg(b), min(b), max(b) with no
    GROUP BY keys: one KDS_FORMAT_ROW tuple, equal to the oracle's and to
    the column arrays.  max(b) is the maximum (the reference's no-group
    global path takes an atomic minimum there, cuda_gpupreagg.cu:524-526).
    The float sum of b (N(0,1) terms, cancelling) is also within 1e-12
    relative of the exactly rounded sum (math.fsum)."""
    import math
    import struct
    tbl, sess, _, expect, meta = C.scan_nogroup(nrows=nrows)
    chunks = tbl.block_chunks(pages_per_chunk=ppc)
    final, st, res = run_gpu(device, sess, chunks, kernel=kernel)
    assert st["nitems_in"] == meta["nitems_in"]
    assert bytes(final)[24:25] == b"r" and struct.unpack_from("<I", bytes(final), 40)[0] == 0
    got = F.decode_kds_final(final, sess)
    assert F.compare_groups(got, expect) == []
    ofinal, _ = run_oracle(sess, chunks)
    want = F.decode_kds_final(ofinal, sess)
    assert F.compare_groups(got, want) == []
    g = got[()]
    assert g[:4] == want[()][:4]                    # integer and numeric states exact
    b, bnull, a = tbl.col("b").values, tbl.col("b").nulls, tbl.col("a").values
    exact = math.fsum(b[(a < 300) & ~bnull].tolist())
    assert abs(g[4][1] - exact) <= 1e-12 * abs(exact)
    assert res["final_nitems"] == 1


def test_no_group_by_no_rows(device, kernel):
    tbl, sess, _, expect, meta = C.scan_nogroup(nrows=10_000, a_limit=0)
    final, st, res = run_gpu(device, sess, tbl.block_chunks(), kernel=kernel)
    assert st["nitems_in"] == 0
    assert F.decode_kds_final(final, sess) == {}


@pytest.mark.parametrize("nrows,ppc", [(40_000, 60), (300_000, 700)])
def test_long_varlena_parity(device, kernel, nrows, ppc):
    """Text group keys of 1..300 bytes (4-byte varlena headers above 126
    bytes, aligned to 4 in the tuple) and numeric(18,4) values in the
    short, NUMERIC_LONG and 4-byte-header long forms, summed and averaged:
    equal to the oracle and to the column arrays."""
    tbl, sess, _, expect, meta = C.long_varlena_groupby(nrows=nrows)
    chunks = tbl.block_chunks(pages_per_chunk=ppc)
    final, st, res = run_gpu(device, sess, chunks, kernel=kernel)
    assert st["nitems_raw"] == meta["nitems_raw"] and st["nitems_in"] == meta["nitems_in"]
    got = F.decode_kds_final(final, sess)
    assert F.compare_groups(got, expect, rtol=0.0) == []
    ofinal, _ = run_oracle(sess, chunks)
    assert F.compare_groups(got, F.decode_kds_final(ofinal, sess), rtol=0.0) == []


def test_join_long_text_keys_parity(device, kernel):
    """GROUP BY an inner relation's text column whose values are up to 300
    bytes (4-byte headers in the inner MinimalTuples)."""
    fact, sess, km, expect, meta = C.join_groupby(nfact=300_000, ndim1=20_000, ndim2=2_000,
                                                  regions=C.long_strings(40))
    chunks = fact.block_chunks(pages_per_chunk=400)
    final, st, res = run_gpu(device, sess, chunks, km, nrels=2, kernel=kernel)
    assert st["nitems_out"] == meta["nitems_out"]
    got = F.decode_kds_final(final, sess)
    truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    assert F.compare_groups(got, truth) == []
    ofinal, _ = run_oracle(sess, chunks, km)
    assert F.compare_groups(got, F.decode_kds_final(ofinal, sess)) == []

"""Pins the oracle to PG-Strom's own code: hash_any, numeric decode and a
full scan/join/group-by pass evaluated by the reference's host-compiled
expression library over the same chunks and bytecode.  Skipped where
oracle/_ref was not built (it needs the reference sources)."""
import os
import sys

import numpy as np
import pytest

import ref_pin
import xb_configs as C
import xb_final as F
import xb_oracle as O
import xb_producer as P

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import ref_fixtures as G  # noqa: E402

pytestmark = pytest.mark.skipif(not ref_pin.available(), reason="oracle/_ref not built")


def test_hash_any_matches_reference():
    r = np.random.default_rng(11)
    for n in list(range(0, 48)) + [100, 255, 1000]:
        d = r.integers(0, 256, n, dtype=np.uint8).tobytes()
        assert ref_pin.hash_any(d) == P.hash_any(d) == O.hash_bytes(d)


def test_numeric_encoding_matches_reference():
    r = np.random.default_rng(12)
    vals = [0, 1, -1, 5, 10, 100, 9999, 10000, 123456, 999999, -999999, 1000000, 12300]
    vals += list(r.integers(-10**9, 10**9, 200))
    for scale in (0, 2, 4):
        for v in vals:
            got = ref_pin.numeric_decode(P.encode_numeric(int(v), scale))
            assert got is not None
            kind, w, iv = got
            assert kind == 0
            # value == v * 10^-scale
            assert iv * 10 ** (scale - w if scale >= w else 0) == v * 10 ** (w - scale if w > scale else 0)
        blob, offs = P.encode_numeric_array(np.array(vals[:50], dtype=np.int64) % 10**7, scale)
        for i in range(50):
            assert bytes(blob[offs[i]:offs[i + 1]]) == P.encode_numeric(int(vals[i] % 10**7), scale)


@pytest.mark.parametrize("which", ["scan", "join", "nogroup", "wide", "long_varlena", "join_long_text", "arrow",
                                   "arrow_nulls", "filtered", "row_scan", "row_wide"])
def test_oracle_matches_reference_functions(which):
    """The oracle's groups equal those the reference's functions compute
    (rtol=0): heap scan and join, an aggregate without GROUP BY keys, every
    partial-state form (count(x), int and float min/max, float sum, numeric
    avg, stddev, covar), text
    and numeric varlenas with 4-byte headers and the NUMERIC_LONG format,
    text group keys of inner rows longer than 126 bytes, and Arrow columns
    read by ExecLoadVarsOuterArrow (int8 / int4 / float8 / date), also with
    validity bitmaps on every column (NULL keys, NULL filter inputs, NULL
    arguments), heap pages whose line pointers are partly unused, dead
    or redirected, and KDS_FORMAT_ROW outer chunks read by
    ExecLoadVarsMinimalTuple."""
    if which == "scan":
        tbl, sess, km, expect, meta = C.scan_groupby(nrows=60_000)
        chunks = tbl.block_chunks(pages_per_chunk=200)
    elif which == "nogroup":
        tbl, sess, km, expect, meta = C.scan_nogroup(nrows=60_000)
        chunks = tbl.block_chunks(pages_per_chunk=200)
    elif which == "wide":
        tbl, sess, km, expect, meta = C.wide_groupby(nrows=60_000, ngroups=800)
        chunks = tbl.block_chunks(pages_per_chunk=200)
    elif which == "long_varlena":
        tbl, sess, km, expect, meta = C.long_varlena_groupby(nrows=20_000)
        chunks = tbl.block_chunks(pages_per_chunk=100)
    elif which == "join_long_text":
        tbl, sess, km, expect, meta = C.join_groupby(nfact=40_000, ndim1=3000, ndim2=500,
                                                     regions=C.long_strings(40))
        chunks = tbl.block_chunks(pages_per_chunk=200)
    elif which == "arrow":
        chunks, sess, expect, meta = C.arrow_groupby(nrows=60_000, nkeys=5_000, rows_per_chunk=25_000)
        km = None
    elif which == "arrow_nulls":
        # (validity NULLs only: the reference asserts that a row its bitmap
        # marks valid has a value, xpu_common.cu:273)
        chunks, sess, expect, meta = C.arrow_nulls(nrows=60_000, nkeys=500, rows_per_chunk=20_000, short_rows=0)
        km = None
    elif which == "filtered":
        chunks, sess, expect, meta = C.scan_groupby_filtered(nrows=60_000, frac=0.2)
        km = None
    elif which == "row_scan":
        tbl, sess, km, expect, meta = C.scan_groupby(nrows=40_000)
        chunks = tbl.row_chunks(rows_per_chunk=9_000)
    elif which == "row_wide":
        tbl, sess, km, expect, meta = C.wide_groupby(nrows=40_000, ngroups=500)
        chunks = tbl.row_chunks(rows_per_chunk=9_000)
    else:
        tbl, sess, km, expect, meta = C.join_groupby(nfact=60_000, ndim1=3000, ndim2=500)
        chunks = tbl.block_chunks(pages_per_chunk=200)
    res = ref_pin.run(sess, chunks, km)
    assert res["nitems_raw"] == meta["nitems_raw"]
    assert res["nitems_in"] == meta["nitems_in"]
    assert res["nitems_out"] == meta["nitems_out"]
    ref = G.decode_groups(res, sess)
    o = O.Oracle(sess, km)
    for ch in chunks:
        o.exec(ch)
    mine = F.decode_kds_final(o.final(), sess)
    o.close()
    assert F.compare_groups(mine, ref, rtol=0.0) == []


def test_reference_gpu_harness_exports():
    """The reference's sm_100a build and the harness that launches it
    (oracle/Makefile ref_gpu): the fatbin is there and the harness exports
    every entry point its front end binds (running it needs a GPU:
    test_gpu_ref_kernel.py)."""
    import ctypes
    import ref_gpu
    if not ref_gpu.available():
        pytest.skip("oracle/_ref/libref_gpu.so or the fatbin not built")
    assert os.path.getsize(ref_gpu.FATBIN) > 0
    L = ctypes.CDLL(ref_gpu.SO)
    for name in ("rg_open", "rg_session", "rg_exec", "rg_final", "rg_info", "rg_close", "rg_upload", "rg_free"):
        assert hasattr(L, name), name
    ref_gpu.lib()


@pytest.mark.parametrize("which", G.CASES)
def test_golden_vectors_are_current(which):
    """The committed golden vectors (tests/golden/ref_pin_*.json, checked
    against the oracle by test_golden_ref.py on hosts without the reference)
    are what the reference's functions compute today over the same inputs."""
    fx = G.load(f"ref_pin_{which}.json")
    sess, chunks, km, _ = G.case_inputs(which)
    assert G.input_digest(sess, chunks, km) == fx["inputs_sha256"]
    res = ref_pin.run(sess, chunks, km)
    for k in ("nitems_raw", "nitems_in", "nitems_out"):
        assert res[k] == fx[k], k
    assert G.decode_groups(res, sess) == G.decode_groups(fx, sess)


def test_golden_scalars_are_current():
    scal = G.load("ref_scalars.json")
    assert [[d.hex(), ref_pin.hash_any(d)] for d in G.hash_inputs()] == scal["hash_any"]
    for (v, s), row in zip(G.numeric_inputs(), scal["numeric"]):
        kind, w, iv = ref_pin.numeric_decode(P.encode_numeric(v, s))
        assert [v, s, kind, w, str(iv)] == row


@pytest.mark.parametrize("which", G.PROJ_CASES)
def test_projection_matches_reference_functions(which):
    """Projection sessions: every row the oracle forms into kds_dst is, byte
    for byte (row id cut off), a row the reference's kern_estimate_minimal_tuple
    / kern_form_minimal_tuple form for the same scan or join result, with
    NULL bitmaps, varlenas and alignment padding; the committed vectors are
    current."""
    sess, chunks, km, _ = G.case_inputs(which)
    res = ref_pin.run(sess, chunks, km)
    ref = sorted(bytes.fromhex(h) for h in res["rows"])
    o = O.Oracle(sess, km)
    for ch in chunks:
        o.exec(ch)
    mine, _ = o.proj_rows()
    st = o.stats()
    o.close()
    assert res["nitems_out"] == st["nitems_out"] == len(ref)
    assert sorted(mine) == ref
    fx = G.load(f"ref_proj_{which}.json")
    assert G.rows_digest(ref) == fx["rows_sha256"]


def test_counts_only_run_matches():
    """ref_pin.run_counts (the bench's reference arm: no groups written
    out) counts the same rows as the full run, on heap and Arrow chunks."""
    tbl, sess, km, _, _ = C.join_groupby(nfact=30_000, ndim1=2000, ndim2=300)
    chunks = tbl.block_chunks(pages_per_chunk=100)
    full = ref_pin.run(sess, chunks, km)
    assert ref_pin.run_counts(sess, chunks, km) == {k: full[k] for k in ("nitems_raw", "nitems_in", "nitems_out")}
    achunks, asess, _, _ = C.arrow_groupby(nrows=30_000, nkeys=3_000, rows_per_chunk=10_000)
    full = ref_pin.run(asess, achunks)
    assert ref_pin.run_counts(asess, achunks) == {k: full[k] for k in ("nitems_raw", "nitems_in", "nitems_out")}

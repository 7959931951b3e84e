"""The reference's own device executor on the B200: PG-Strom's
kern_gpujoin_main (src/cuda_gpujoin.cu:1050-1279) built for sm_100a from the
reference sources (oracle/Makefile "ref_gpu") and launched as PG-Strom's GPU
service launches it (oracle/ref_gpu.cpp), over the same sessions and chunks
as this repository's kernels.  Its kds_final must hold the groups of the C
oracle and of this repository's path: integer and numeric states exact,
float states within the float tolerance; its row counters must match.  The
reference kernel is the checker here and the baseline of bench.py; nothing
of the product runs it."""
import pytest

import xb_configs as C
import xb_final as F
import xb_oracle as O
import xpu_b200

pytestmark = pytest.mark.gpu

ref_gpu = pytest.importorskip("ref_gpu")


@pytest.fixture(scope="module")
def ref_device(device):
    if not ref_gpu.available():
        pytest.skip("the reference's sm_100a build (oracle/_ref) is not present")
    ref_gpu.open_device(0)
    return device


def _oracle_groups(sess, chunks, km=None):
    o = O.Oracle(sess, km)
    for ch in chunks:
        o.exec(ch)
    want = F.decode_kds_final(o.final(), sess)
    st = o.stats()
    o.close()
    return want, st


def _ref_run(sess, chunks, km=None):
    ptrs = [ref_gpu.upload(ch) for ch in chunks]
    rs = ref_gpu.RefSession(sess, km)
    try:
        rs.exec(ptrs)
        final = rs.final()
        info = rs.info()
    finally:
        rs.close()
        for p in ptrs:
            ref_gpu.free(p)
    return final, info


def test_reference_kernel_scan_groupby(ref_device):
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=200_000, seed_config=91)
    chunks = tbl.block_chunks(pages_per_chunk=512)
    final, info = _ref_run(sess, chunks)
    got = F.decode_kds_final(final, sess)
    want, st = _oracle_groups(sess, chunks)
    assert F.compare_groups(got, want) == []
    assert info["nitems_raw"] == meta["nitems_raw"]
    assert info["nitems_out"] == st["nitems_out"]
    truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
    assert F.compare_groups(got, truth) == []


def test_reference_kernel_join_groupby(ref_device):
    fact, sess, km, expect, meta = C.join_groupby(nfact=300_000, ndim1=20_000, ndim2=1_000, seed_config=92)
    chunks = fact.block_chunks(pages_per_chunk=512)
    final, info = _ref_run(sess, chunks, km)
    got = F.decode_kds_final(final, sess)
    want, _ = _oracle_groups(sess, chunks, km)
    assert F.compare_groups(got, want) == []
    truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    assert F.compare_groups(got, truth) == []
    # the same groups as this repository's kernel
    s = xpu_b200.Session(ref_device, sess, km, 2)
    try:
        for ch in chunks:
            s.exec(ch)
        mine, _ = s.final()
    finally:
        s.close()
    assert F.compare_groups(F.decode_kds_final(mine, sess), got) == []

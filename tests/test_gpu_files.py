"""Chunks from files and chunks resident across sessions, on the GPU: a
heap relation file's chunks placed in the library's resident chunk cache
serve two sessions (the second without any upload), pinned chunks survive
eviction and unpinned ones go least recently used first; an Arrow IPC
file with a dictionary-encoded text column is grouped by that column on
both kernels, equal to the oracle and the arrays."""
import os

import pytest

import xb_configs as C
import xb_files as XF
import xb_final as F
import xpu_b200
from test_files import arrow_dict_case

pytestmark = pytest.mark.gpu

TABLE = 0x7AB1E


@pytest.fixture(params=["jit", "vm"])
def kernel(request, monkeypatch):
    monkeypatch.setenv("XPU_B200_JIT", "1" if request.param == "jit" else "0")
    return request.param


def _run_cached(device, sess, ptrs):
    s = xpu_b200.Session(device, sess)
    try:
        for p in ptrs:
            s.exec(p, on_device=True)
        final, _ = s.final()
    finally:
        s.close()
    return F.decode_kds_final(final, sess)


def test_heap_file_chunks_resident_across_sessions(device, tmp_path):
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=400_000, seed_config=32)
    path = str(tmp_path / "16385")
    XF.write_heap_relation(tbl, path)
    chunks = XF.heap_file_chunks(tbl, path, pages_per_chunk=1024)
    truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
    before = device.chunk_cache()
    ptrs = [device.chunk_put(TABLE, i, ch) for i, ch in enumerate(chunks)]
    try:
        assert device.chunk_cache() >= before + sum(c.nbytes for c in chunks)
        assert F.compare_groups(_run_cached(device, sess, ptrs), truth) == []
        # a second query finds every chunk resident: the same addresses
        again = [device.chunk_get(TABLE, i) for i in range(len(chunks))]
        assert again == ptrs
        assert F.compare_groups(_run_cached(device, sess, again), truth) == []
        for p in again:
            assert device.chunk_release(p)
        assert device.chunk_get(TABLE, len(chunks)) is None
        # pinned chunks survive a budget of nothing; released ones leave
        device.chunk_cache(0)
        assert device.chunk_get(TABLE, 0) == ptrs[0]
        device.chunk_release(ptrs[0])
    finally:
        for p in ptrs:
            device.chunk_release(p)
        device.chunk_cache(0)
        device.chunk_cache(64 << 30)
    assert device.chunk_get(TABLE, 0) is None


def test_arrow_ipc_dictionary_column_on_the_device(device, kernel, tmp_path):
    path, sess, expect, nin = arrow_dict_case(tmp_path, nrows=300_000, seed=33)
    chunks, _ = XF.arrow_ipc_chunks(path)
    s = xpu_b200.Session(device, sess)
    try:
        n = 0
        for ch in chunks:
            n += s.exec(ch)["nitems_in"]
        final, _ = s.final()
    finally:
        s.close()
    assert n == nin
    assert F.compare_groups(F.decode_kds_final(final, sess), expect) == []


@pytest.mark.parametrize("try_direct", [True, False])
def test_heap_file_read_direct_into_device(device, tmp_path, try_direct):
    """xpuB200ChunkReadDirect: each chunk's header from host memory and its
    heap pages from the relation file into device memory, then the chunks
    run from the device: the same bytes as heap_file_chunks and the same
    groups as the truth.  try_direct without XPU_B200_CUFILE=1 leaves
    libcufile alone and reads every page through the bounce buffer (every
    page counted once)."""
    assert os.environ.get("XPU_B200_CUFILE") != "1"
    import numpy as np
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=300_000, seed_config=35)
    path = str(tmp_path / "16387")
    XF.write_heap_relation(tbl, path)
    want = XF.heap_file_chunks(tbl, path, pages_per_chunk=512)
    plan = XF.heap_file_iovec(tbl, path, pages_per_chunk=512, io_pages=96)
    truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
    bases, ptrs = [], []
    try:
        for ch, w in zip(plan, want):
            size = ch["length"] + XF.IO_PAGE
            base = device.alloc(size)
            bases.append(base)
            # the header ends on a page boundary of device memory
            gap = (-(base + ch["base_offset"])) % XF.IO_PAGE
            dptr = base + gap
            nd, nv = device.read_direct(path, ch["head"], ch["base_offset"], ch["iov"], dptr,
                                        size - gap, try_direct=try_direct)
            assert nd + nv == (ch["length"] - ch["base_offset"]) // XF.IO_PAGE
            assert nd == 0
            got = np.frombuffer(device.download(dptr, ch["length"]), dtype=np.uint8)
            assert got.tobytes() == w.tobytes()
            ptrs.append(dptr)
        assert F.compare_groups(_run_cached(device, sess, ptrs), truth) == []
    finally:
        for b in bases:
            device.free(b)


def test_read_direct_rejects_a_chunk_past_the_buffer(device, tmp_path):
    tbl, sess, _, expect, meta = C.scan_groupby(nrows=20_000, seed_config=36)
    path = str(tmp_path / "16388")
    XF.write_heap_relation(tbl, path)
    ch = XF.heap_file_iovec(tbl, path, pages_per_chunk=64)[0]
    base = device.alloc(ch["length"])
    try:
        with pytest.raises(xpu_b200.XpuB200Error, match="past the device buffer"):
            device.read_direct(path, ch["head"], ch["base_offset"], ch["iov"], base, ch["length"] - 1)
    finally:
        device.free(base)

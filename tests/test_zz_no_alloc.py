"""xpuB200FinalNoAlloc: kds_final for callers that cannot allocate GPU memory.

Some callers of this library cannot call cudaMalloc: a GPU service that has
reserved the device's memory up front and hands out pieces of its own pool,
or one that must not call cudaMalloc / cudaFree while other sessions' kernels
run (cudaFree waits for the whole device).  This entry point writes kds_final
into memory the caller already owns and keeps its work arrays in a fixed
array inside the library.  Its output must be the same groups, with the same
sizes, as xpuB200Final's, call after call, although every call reuses the
array that the previous call left behind.

The file is named so that pytest collects it after every other test file.
"""
import ctypes
import struct

import numpy as np
import pytest

import xb_configs as C
import xb_final as F
import xpu_b200

pytestmark = pytest.mark.gpu


def _final_no_alloc(sess, dptr, nbytes):
    """Calls the entry point; returns (rc, required bytes, results, message)."""
    L = xpu_b200.lib()
    fn = L.xpuB200FinalNoAlloc
    fn.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_uint64, ctypes.POINTER(ctypes.c_uint64),
                   ctypes.c_void_p, ctypes.POINTER(xpu_b200.KernErrorbuf)]
    fn.restype = ctypes.c_int
    req = ctypes.c_uint64()
    res = xpu_b200.results_buffer(sess.nrels)
    res[92:96] = np.frombuffer(np.uint32(sess.nrels).tobytes(), dtype=np.uint8)
    e = xpu_b200.KernErrorbuf()
    rc = fn(sess.h, ctypes.c_void_p(dptr), nbytes, ctypes.byref(req), xpu_b200._ptr(res), ctypes.byref(e))
    return rc, req.value, xpu_b200.parse_results(res), e.message.decode(errors="replace")


def _no_alloc_final_bytes(sess):
    """kds_final through the entry point, into a device buffer owned by the test."""
    import torch
    rc, need, _, msg = _final_no_alloc(sess, 0, 0)
    assert rc == 0, msg
    out = torch.zeros(need, dtype=torch.uint8, device="cuda:0")
    torch.cuda.synchronize()
    rc, need2, res, msg = _final_no_alloc(sess, out.data_ptr(), need)
    assert rc == 0, msg
    assert need2 == need
    return out.cpu().numpy(), res


def _layout(buf):
    """(bytes with the hash-chain links blanked, {slot: set of item offsets}).
    Items enter their slot's chain concurrently, so only the chains' order
    may differ between two calls; every other byte must be the same."""
    b = np.array(buf, dtype=np.uint8, copy=True)
    length, _usage, nitems = struct.unpack_from("<QQI", b, 0)
    nslots = struct.unpack_from("<I", b, 40)[0]
    nr_colmeta = struct.unpack_from("<I", b, 68)[0]
    head = (72 + 168 * nr_colmeta + 7) & ~7          # KDS_HEAD_LENGTH
    slots = np.frombuffer(b[head:head + 8 * nslots].tobytes(), dtype=np.uint64)
    chains = {}
    for slot in np.flatnonzero(slots).tolist():
        off = int(slots[slot])
        seen = set()
        while off:
            item = length - off
            assert item not in seen
            seen.add(item)
            off = struct.unpack_from("<Q", b, item)[0]
        chains[slot] = seen
    assert sum(len(v) for v in chains.values()) == nitems
    b[head:head + 8 * nslots] = 0
    for items in chains.values():
        for item in items:
            b[item:item + 8] = 0
    return b.tobytes(), chains


def _open(device, which):
    if which == "join":
        fact, sess, km, expect, _ = C.join_groupby(nfact=60_000, ndim1=3_000, ndim2=400)
        s = xpu_b200.Session(device, sess, km, 2)
        for ch in fact.block_chunks(pages_per_chunk=100):
            s.exec(ch)
        truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    else:
        tbl, sess, _, expect, _ = C.scan_groupby(nrows=40_000)
        s = xpu_b200.Session(device, sess)
        for ch in tbl.block_chunks(pages_per_chunk=64):
            s.exec(ch)
        truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
    return s, sess, truth


def test_final_without_allocation_matches_final(device):
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device for the output buffer")
    s_join, sess_join, truth_join = _open(device, "join")
    s_scan, sess_scan, truth_scan = _open(device, "scan")
    try:
        want, want_res = s_join.final()
        want_groups = F.decode_kds_final(want, sess_join)
        assert F.compare_groups(want_groups, truth_join) == []

        # two calls in a row on the same session, with another session's call
        # in between so that the shared work array holds other data
        first, res1 = _no_alloc_final_bytes(s_join)
        other, _ = _no_alloc_final_bytes(s_scan)
        second, res2 = _no_alloc_final_bytes(s_join)
        want_bytes, want_chains = _layout(want)
        for got, res in ((first, res1), (second, res2)):
            assert got.nbytes == want.nbytes
            assert res["final_nitems"] == want_res["final_nitems"]
            assert F.compare_groups(F.decode_kds_final(got, sess_join), want_groups) == []
            # byte for byte the same buffer, up to the order of hash chains
            got_bytes, got_chains = _layout(got)
            assert got_chains == want_chains
            assert got_bytes == want_bytes
        assert F.compare_groups(F.decode_kds_final(other, sess_scan), truth_scan) == []
    finally:
        s_join.close()
        s_scan.close()


def test_final_without_allocation_rejects_large_group_tables(device):
    # 100,000 estimated groups size the group table at 524,288 slots: more
    # work space than the fixed array holds
    chunks, sess, _, _ = C.arrow_groupby(nrows=100_000, nkeys=100_000, rows_per_chunk=100_000,
                                         with_expect=False)
    s = xpu_b200.Session(device, sess)
    try:
        rc, _, _, msg = _final_no_alloc(s, 0, 0)
        assert rc == ord("E")
        assert "use xpuB200Final" in msg
    finally:
        s.close()

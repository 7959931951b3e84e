"""Device projection on the GPU (xpuB200ExecTaskDst): every chunk's
kds_dst holds exactly the oracle's rows for that chunk, byte for byte
apart from the row ids (rows are placed in whatever order the warps claim
space, as in the reference), with the reference's per-row space
accounting.  Runs on both kernels, like test_gpu_parity.py."""
import pytest

import xb_configs as C
import xb_oracle as O
import xb_rows as RW
import xpu_b200

pytestmark = pytest.mark.gpu

@pytest.fixture(params=["jit", "vm"])
def kernel(request, monkeypatch):
    monkeypatch.setenv("XPU_B200_JIT", "1" if request.param == "jit" else "0")
    return request.param


def _check_kernel(s, kernel):
    info = s.info()
    assert set(info["kernels"].values()) == {kernel}, f"{info['kernels']}: {info['jit_msg']}"


def _compare_chunk(dst, o, dst_size):
    """kds_dst of one chunk against the oracle's rows of the same chunk."""
    head, rows = RW.decode_kds_rows(dst)
    want, want_usage = o.proj_rows(reset=True)
    assert head["format"] == "r"
    assert head["length"] == dst_size
    assert head["nitems"] == len(want)
    assert head["usage"] == want_usage
    assert [r[1] for r in rows] == list(range(len(rows)))     # row id = row index slot
    assert sorted(r[0] for r in rows) == sorted(want)
    return rows


def _run(device, kernel, sess, chunks, kmrels=None, nrels=0, dst_size=1 << 22):
    s = xpu_b200.Session(device, sess, kmrels, nrels)
    o = O.Oracle(sess, kmrels)
    values, retries = [], 0
    tot = {"nitems_raw": 0, "nitems_in": 0, "nitems_out": 0}
    try:
        for ch in chunks:
            dst, res, retried = s.exec_dst(ch, dst_size)
            retries += retried
            o.exec(ch)
            rows = _compare_chunk(dst, o, dst.nbytes)
            values += [tuple(r[2]) for r in rows]
            for k in tot:
                tot[k] += res[k]
        _check_kernel(s, kernel)
    finally:
        s.close()
        o.close()
    return values, tot, retries


@pytest.mark.parametrize("nrows,ppc,margin", [(20_000, 64, 0), (300_000, 1000, 16)])
def test_scan_projection_parity(device, kernel, nrows, ppc, margin):
    tbl, sess, expect, meta = C.scan_projection(nrows=nrows, htup_margin=margin)
    values, tot, _ = _run(device, kernel, sess, tbl.block_chunks(pages_per_chunk=ppc))
    assert tot["nitems_raw"] == meta["nitems_raw"]
    assert tot["nitems_out"] == meta["nitems_out"] == len(values)
    assert sorted(v[0] for v in values) == sorted(expect)
    for v in values:
        assert (v[1], v[2], v[4]) == expect[v[0]]


@pytest.mark.parametrize("copies,stride,miss", [(1, 1, 0.0), (3, 7, 0.2), (2, 13, 0.1)])
def test_join_projection_parity(device, kernel, copies, stride, miss):
    fact, sess, km, meta = C.join_projection(nfact=60_000, dim1_copies=copies, key_stride=stride,
                                             miss_frac=miss)
    values, tot, _ = _run(device, kernel, sess, fact.block_chunks(pages_per_chunk=100), km, 2)
    assert tot["nitems_out"] == meta["nitems_out"]
    assert sorted(values) == meta["rows"]


def test_projection_no_space_then_retry(device, kernel):
    # 4 KiB holds a few dozen rows: every chunk first answers SUSPEND_NO_SPACE
    # with the size it needs, and the retry with that size returns all rows
    tbl, sess, expect, meta = C.scan_projection(nrows=40_000)
    values, tot, retries = _run(device, kernel, sess, tbl.block_chunks(pages_per_chunk=100), dst_size=4096)
    assert retries == len(tbl.block_chunks(pages_per_chunk=100))
    assert sorted(v[0] for v in values) == sorted(expect)


def test_projection_into_device_memory(device, kernel):
    torch = pytest.importorskip("torch")
    import ctypes
    tbl, sess, expect, _ = C.scan_projection(nrows=20_000)
    s = xpu_b200.Session(device, sess)
    o = O.Oracle(sess)
    L = xpu_b200.lib()
    try:
        out = torch.zeros(1 << 21, dtype=torch.uint8, device="cuda:0")
        torch.cuda.synchronize()
        for ch in tbl.block_chunks(pages_per_chunk=64):
            res = xpu_b200.results_buffer(0)
            e = xpu_b200.KernErrorbuf()
            req = ctypes.c_uint64()
            rc = L.xpuB200ExecTaskDst(s.h, xpu_b200._ptr(ch), 0, ctypes.c_void_p(out.data_ptr()), out.numel(), 1,
                                      ctypes.byref(req), xpu_b200._ptr(res), ctypes.byref(e))
            assert rc == 0, e.message
            o.exec(ch)
            _compare_chunk(out.cpu().numpy(), o, out.numel())
        _check_kernel(s, kernel)
    finally:
        s.close()
        o.close()


def test_exec_task_refuses_projection_session(device):
    tbl, sess, _, _ = C.scan_projection(nrows=2_000)
    s = xpu_b200.Session(device, sess)
    try:
        with pytest.raises(xpu_b200.XpuB200Error, match="xpuB200ExecTaskDst"):
            s.exec(tbl.block_chunks(pages_per_chunk=64)[0])
    finally:
        s.close()

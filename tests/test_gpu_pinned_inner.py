"""Pinned inner buffers on the GPU: a scan of a dimension table projects
its rows, each carrying the join's inner hash (u.proj.hash), into a
KDS_FORMAT_HASH kds_dst; the chunks' buffers are rebuilt into one hashed
inner buffer on the device (xpuB200InnerRebuild), or split into hash
partitions, and the rebuilt buffer serves as the inner relation of the
fact-dim1-dim2 join, whose groups must equal the generator's truth.  Rows
are compared with the oracle's byte for byte apart from row ids; every
row must be reachable through the hash chain of its slot."""
import struct

import numpy as np
import pytest

import xb_configs as C
import xb_final as F
import xb_oracle as O
import xb_rows as RW
import xpu_b200
from xb_producer import kern_multirels

pytestmark = pytest.mark.gpu

NSLOTS = 4096


def _chains(buf):
    """(row images without row ids, row ids) of a KDS_FORMAT_HASH buffer,
    checking that each row is on the chain of its hash slot exactly once"""
    b = bytes(buf)
    head, rows = RW.decode_kds_rows(b)
    assert head["format"] == "h"
    length, nitems = head["length"], head["nitems"]
    nslots, = struct.unpack_from("<I", b, 40)
    ncol, = struct.unpack_from("<I", b, 68)
    hl = (72 + 168 * ncol + 7) & ~7
    slots = np.frombuffer(b, dtype=np.uint64, count=nslots, offset=hl)
    on_chain = {}
    for k in range(nslots):
        off = int(slots[k])
        steps = 0
        while off:
            item = length - off
            t = item + 8
            h, = struct.unpack_from("<I", b, t + 4)
            assert h % nslots == k
            on_chain[t] = on_chain.get(t, 0) + 1
            off, = struct.unpack_from("<Q", b, item)
            steps += 1
            assert steps <= nitems
    rowidx = np.frombuffer(b, dtype=np.uint64, count=nitems, offset=hl + 8 * nslots)
    ts = sorted(length - int(x) for x in rowidx)
    assert sorted(on_chain) == ts and all(v == 1 for v in on_chain.values())
    return [r[0] for r in rows], [r[1] for r in rows]


def _template(sess, length, nslots=NSLOTS):
    """empty KDS_FORMAT_HASH buffer with the projection's kds_dst columns"""
    off, = struct.unpack_from("<I", sess, 128)
    ncol, = struct.unpack_from("<I", sess, off + 68)
    hl = (72 + 168 * ncol + 7) & ~7
    buf = np.zeros(length, dtype=np.uint8)
    buf[:hl] = np.frombuffer(bytes(sess[off:off + hl]), dtype=np.uint8)
    struct.pack_into("<QQI", buf, 0, length, 0, 0)
    struct.pack_into("<I", buf, 40, nslots)
    return buf


def _project(device, ps, dim1):
    s = xpu_b200.Session(device, ps)
    o = O.Oracle(ps)
    outs, oracle_rows = [], []
    try:
        for ch in dim1.block_chunks(pages_per_chunk=40):
            dst, res, _ = s.exec_dst(ch, 1 << 22)
            o.exec(ch)
            want, want_usage = o.proj_rows(reset=True)
            imgs, ids = _chains(dst)
            head, _ = RW.decode_kds_rows(dst)
            assert head["nitems"] == len(want)
            assert head["usage"] == want_usage + 8 * len(want)       # kern_hashitem.next per row
            assert sorted(ids) == list(range(len(want)))
            assert sorted(imgs) == sorted(want)
            assert "vm" in set(s.info()["kernels"].values())
            outs.append(dst)
            oracle_rows += want
    finally:
        s.close()
        o.close()
    return outs, oracle_rows


def test_pinned_inner_rebuild_partition_and_join(device):
    fact, sess, km, expect, meta = C.join_groupby(nfact=300_000, ndim1=20_000, ndim2=700, seed_config=31)
    dims = meta["dims"]
    ps = C.pinned_dim1_session(nslots=NSLOTS)
    outs, all_rows = _project(device, ps, dims["dim1"])
    assert len(all_rows) == 20_000
    # the hash every row carries is the join's inner hash of its pk
    cols = RW.kds_columns(bytes(_template(ps, 1 << 16)))
    want_h = dict(zip(dims["pk1"].tolist(), C.host_join_hash_int4(dims["pk1"]).tolist()))
    for img in all_rows[:2000]:
        pk, _ = RW.decode_tuple(img + b"\0" * 8, 0, cols)
        assert struct.unpack_from("<I", img, 4)[0] == want_h[pk]
    srcs = [device.upload(o, align_pages=False) for o in outs]
    bases = [b for b, _ in srcs]
    try:
        # every chunk's rows into one buffer
        length = 4 << 20
        dbase, dptr = device.upload(_template(ps, length), align_pages=False)
        bases.append(dbase)
        for _, p in srcs:
            device.inner_rebuild(dptr, p)
        inner = device.download(dptr, length)
        imgs, ids = _chains(inner)
        assert sorted(imgs) == sorted(all_rows)
        assert sorted(ids) == list(range(len(all_rows)))
        # three hash partitions hold every row once
        parts = []
        for r in range(3):
            pb, pp = device.upload(_template(ps, 2 << 20), align_pages=False)
            bases.append(pb)
            for _, p in srcs:
                device.inner_rebuild(pp, p, divisor=3, remainder=r)
            pimgs, _ = _chains(device.download(pp, 2 << 20))
            assert all(struct.unpack_from("<I", x, 4)[0] % 3 == r for x in pimgs)
            parts += pimgs
        assert sorted(parts) == sorted(all_rows)
        # too small a destination: the bytes it needs, and no partial success
        sb, sp = device.upload(_template(ps, 64 << 10), align_pages=False)
        bases.append(sb)
        with pytest.raises(xpu_b200.XpuB200Error, match="needs"):
            for _, p in srcs:
                device.inner_rebuild(sp, p)
        # the rebuilt buffer as the join's dim1
        kmr = kern_multirels([inner, dims["dim2"].hash_kds(C.host_join_hash_int4(dims["pk2"]))])
        for jit in ("1", "0"):
            import os
            os.environ["XPU_B200_JIT"] = jit
            try:
                s = xpu_b200.Session(device, sess, kmr, 2)
                for ch in fact.block_chunks(pages_per_chunk=300):
                    s.exec(ch)
                final, _ = s.final()
                s.close()
            finally:
                os.environ.pop("XPU_B200_JIT", None)
            truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
            assert F.compare_groups(F.decode_kds_final(final, sess), truth) == []
    finally:
        for b in bases:
            device.free(b)

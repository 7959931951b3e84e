"""The device side of the hash-partitioned multi-GPU merge, with three
ranks emulated on one GPU: each rank's groups are split by hash % 3 on the
device (xpuB200FinalParts, one buffer of three KDS_FORMAT_HASH parts) and
rank r merges part r of every rank straight from device memory
(xpuB200MergeFinal on device), as it would from a peer's memory.  Every
group must end on exactly one rank with the states of one session over all
chunks; the exchange of the bytes between processes is tested with gloo
ranks in test_multirank.py."""
import struct

import pytest

import xb_configs as C
import xb_exchange as X
import xb_final as F
import xpu_b200

pytestmark = pytest.mark.gpu

WORLD = 3


def _exchange(device, sess, chunks, km=None, nrels=0):
    """Three emulated ranks, each with its share of the chunks; every rank
    splits its groups on the device and rank r merges part r of all."""
    sessions, bufs = [], []
    try:
        for r in range(WORLD):
            s = xpu_b200.Session(device, sess, km, nrels)
            sessions.append(s)
            for ch in chunks[r::WORLD]:
                s.exec(ch)
            bufs.append(X.final_parts(device, s, WORLD))
        for base, offs in bufs:
            assert offs[0] == 0 and all(o % 256 == 0 for o in offs)
            for r in range(WORLD):
                p = device.download(base + offs[r], offs[r + 1] - offs[r])
                length, = struct.unpack_from("<Q", p, 0)
                assert bytes(p[24:25]) == b"h" and length <= len(p)
                p = p[:length]
                # every tuple of part r hashes to r
                n, = struct.unpack_from("<I", p, 16)
                ncol, = struct.unpack_from("<I", p, 68)
                nslots, = struct.unpack_from("<I", p, 40)
                hl = (72 + 168 * ncol + 7) & ~7
                for i in range(n):
                    off, = struct.unpack_from("<Q", p, hl + 8 * nslots + 8 * i)
                    h, = struct.unpack_from("<I", p, length - off + 4)
                    assert h % WORLD == r
        merged = {}
        for r in range(WORLD):
            m = xpu_b200.Session(device, sess, km, nrels)
            try:
                for base, offs in bufs:
                    m.merge_final(base + offs[r], on_device=True)
                f, _ = m.final()
            finally:
                m.close()
            d = F.decode_kds_final(f, sess) if f is not None else {}
            assert not (set(d) & set(merged))              # a group lives on one rank only
            merged.update(d)
        return merged
    finally:
        for s in sessions:
            s.close()
        for base, _ in bufs:
            device.free(base)


def test_exchange_wide_groupby(device):
    tbl, sess, _, expect, meta = C.wide_groupby(nrows=300_000, ngroups=5000, seed_config=61)
    chunks = tbl.block_chunks(pages_per_chunk=128)
    merged = _exchange(device, sess, chunks)
    assert F.compare_groups(merged, expect) == []


def test_exchange_arrow_many_groups(device):
    chunks, sess, expect, meta = C.arrow_groupby(nrows=900_000, nkeys=300_000, rows_per_chunk=100_000,
                                                 seed_config=62)
    merged = _exchange(device, sess, chunks)
    assert F.compare_groups(merged, expect) == []


def test_exchange_join_text_keys(device):
    fact, sess, km, expect, meta = C.join_groupby(nfact=150_000, ndim1=5000, ndim2=700, seed_config=63)
    chunks = fact.block_chunks(pages_per_chunk=100)
    merged = _exchange(device, sess, chunks, km, 2)
    truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    assert F.compare_groups(merged, truth) == []

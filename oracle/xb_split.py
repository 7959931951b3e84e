"""
Host restatement of the exchange step of a multi-GPU pre-aggregation:
a kds_final split into hash partitions (what xpuB200FinalParts writes on
the device) and the merge of received partial states (what
xpuB200MergeFinal adds into a group table).  TEST INFRASTRUCTURE ONLY:
used by tests/ as the checker of the exchange path; the product never
imports it.  The state arithmetic follows the reference's final merge
(kern_gpupreagg_final_merge, cuda_gpupreagg.cu:2331-2432): counts and
sums add, minima and maxima keep the extreme of the valid ones.
"""
import struct

import numpy as np

KAGG_MIN = (302, 303, 304)
KAGG_MAX = (402, 403, 404)


def _head(buf):
    length, usage, nitems = struct.unpack_from("<QQI", buf, 0)
    nslots, = struct.unpack_from("<I", buf, 40)
    nr_colmeta, = struct.unpack_from("<I", buf, 68)
    hl = (72 + 168 * nr_colmeta + 7) & ~7
    return length, nitems, nslots, hl


def split_kds_final(buf, nparts):
    """KDS_FORMAT_HASH parts of a kds_final by tuple hash % nparts: each part
    a kds_final of its own (header, hash slots, row index, the tuples'
    kern_hashitems), None when no group falls into it."""
    b = bytes(buf)
    length, nitems, nslots, hl = _head(b)
    rowidx = np.frombuffer(b, dtype=np.uint64, count=nitems, offset=hl + 8 * nslots)
    items = [[] for _ in range(nparts)]
    for i in range(nitems):
        t = length - int(rowidx[i])                    # kern_tupitem
        t_len, h = struct.unpack_from("<II", b, t)
        items[h % nparts].append((h, b[t:t + t_len]))
    parts = []
    for lst in items:
        if not lst:
            parts.append(None)
            continue
        n = len(lst)
        ns = 20000 if n <= 5000 else (20000 + 2 * n if n <= 4_000_000 else 8020000 + n)
        sizes = [(8 + len(tup) + 7) & ~7 for _, tup in lst]
        plen = hl + 8 * ns + 8 * n + sum(sizes)
        out = bytearray(plen)
        out[:hl] = b[:hl]
        struct.pack_into("<QQI", out, 0, plen, sum(sizes), n)
        out[24] = ord("h")
        struct.pack_into("<I", out, 40, ns)
        pos = hl + 8 * ns + 8 * n
        for i, ((h, tup), sz) in enumerate(zip(lst, sizes)):
            slot = h % ns
            prev, = struct.unpack_from("<Q", out, hl + 8 * slot)
            struct.pack_into("<Q", out, pos, prev)                  # kern_hashitem.next
            out[pos + 8:pos + 8 + len(tup)] = tup
            struct.pack_into("<Q", out, hl + 8 * slot, plen - pos)
            struct.pack_into("<Q", out, hl + 8 * ns + 8 * i, plen - (pos + 8))
            pos += sz
        parts.append(np.frombuffer(bytes(out), dtype=np.uint8))
    return parts


def tuple_hashes(buf):
    """The hash of every group tuple of a kds_final."""
    b = bytes(buf)
    length, nitems, nslots, hl = _head(b)
    rowidx = np.frombuffer(b, dtype=np.uint64, count=nitems, offset=hl + 8 * nslots)
    return [struct.unpack_from("<I", b, length - int(r) + 4)[0] for r in rowidx]


def merge_states(actions, into, states):
    """states (decoded by xb_final.decode_kds_final) added into 'into'."""
    out = []
    for act, a, b in zip(actions, into, states):
        if isinstance(a, int):
            out.append(a + b)
        elif act in KAGG_MIN or act in KAGG_MAX:
            if not a[0]:
                out.append(b)
            elif not b[0]:
                out.append(a)
            else:
                out.append((1, min(a[1], b[1]) if act in KAGG_MIN else max(a[1], b[1])))
        else:
            out.append(tuple(x + y if i < 2 else x for i, (x, y) in enumerate(zip(a, b))))
    return out

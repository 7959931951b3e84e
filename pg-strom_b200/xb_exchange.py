"""
Multi-GPU merge of partial-aggregation results by hash partitioning: each
rank splits its kds_final into one KDS_FORMAT_HASH part per rank by
hash % world on its GPU (xpuB200InnerRebuild), the parts are exchanged
all-to-all through torch.distributed (NCCL over NVLink between GPUs, gloo
between CPU processes), and each rank merges the parts it received into a
fresh session of the same plan (xpuB200MergeFinal), so that every group
ends on exactly one rank.  This is the exchange step of a multi-GPU
GpuPreAgg whose groups are too many to gather on one GPU; the reference
merges every GPU's kds_final into the first one instead
(__gpuservHandleGpuPreAggFinal, gpu_service.c:5442-5518).
"""
import struct

import numpy as np


def _final_template(session: bytes):
    """(header bytes, header length) of the session's kds_final definition"""
    off, = struct.unpack_from("<I", session, 156)
    ncol, = struct.unpack_from("<I", session, off + 68)
    hl = (72 + 168 * ncol + 7) & ~7
    return bytes(session[off:off + hl]), hl


def empty_final_part(session: bytes, length: int, nslots: int) -> np.ndarray:
    """An empty KDS_FORMAT_HASH buffer with the columns of the session's
    kds_final: length bytes, nslots zeroed hash slots."""
    head, hl = _final_template(session)
    buf = np.zeros(length, dtype=np.uint8)
    buf[:hl] = np.frombuffer(head, dtype=np.uint8)
    struct.pack_into("<QQI", buf, 0, length, 0, 0)
    buf[24] = ord("h")
    struct.pack_into("<I", buf, 40, nslots)
    return buf


def split_final(dev, session: bytes, final: np.ndarray, nparts: int):
    """The groups of one kds_final split into nparts KDS_FORMAT_HASH parts
    by hash % nparts, on the device; returns host copies (None for an empty
    part)."""
    if final is None:
        return [None] * nparts
    length = int(struct.unpack_from("<Q", final, 0)[0])
    nitems = int(struct.unpack_from("<I", final, 16)[0])
    nslots = max(1024, 2 * (nitems // nparts + 1))
    base, src = dev.upload(final, align_pages=False)
    parts, bases = [], [base]
    try:
        for r in range(nparts):
            _, hl = _final_template(session)
            plen = (hl + 8 * nslots + length + 7) & ~7      # every row could fall here
            pb, pp = dev.upload(empty_final_part(session, plen, nslots), align_pages=False)
            bases.append(pb)
            used = dev.inner_rebuild(pp, src, divisor=nparts, remainder=r)
            part = dev.download(pp, plen)
            n = int(struct.unpack_from("<I", part, 16)[0])
            if n == 0:
                parts.append(None)
                continue
            # cut the unused middle: header, slots, row index, then the rows
            usage = int(struct.unpack_from("<Q", part, 8)[0])
            head = hl + 8 * nslots + 8 * n
            out = np.concatenate([part[:head], part[plen - usage:]])
            struct.pack_into("<Q", out, 0, len(out))
            assert used == len(out)
            parts.append(out)
    finally:
        for b in bases:
            dev.free(b)
    return parts


def alltoall_bytes(parts, rank, world, device=None):
    """parts[r] (bytes-like or None) goes to rank r; returns the parts every
    rank sent to this one, in rank order.  Two exchanges: the sizes, then
    the bytes with uneven splits (all_to_all_single)."""
    import torch
    import torch.distributed as dist
    sizes = [0 if p is None else len(p) for p in parts]
    dev = device if device is not None else "cpu"
    send_n = torch.tensor(sizes, dtype=torch.int64, device=dev)
    recv_n = torch.empty(world, dtype=torch.int64, device=dev)
    dist.all_to_all_single(recv_n, send_n)
    recv_sizes = recv_n.cpu().tolist()
    blob = np.concatenate([np.asarray(p, dtype=np.uint8) for p in parts if p is not None]) \
        if any(sizes) else np.zeros(0, dtype=np.uint8)
    send = torch.from_numpy(blob).to(dev)
    recv = torch.empty(sum(recv_sizes), dtype=torch.uint8, device=dev)
    dist.all_to_all_single(recv, send, output_split_sizes=recv_sizes, input_split_sizes=sizes)
    recv = recv.cpu().numpy()
    out, pos = [], 0
    for n in recv_sizes:
        out.append(recv[pos:pos + n].copy() if n else None)
        pos += n
    return out


def merge_parts(dev, session: bytes, parts, kmrels=None, nrels=0):
    """A fresh session of the plan with every received part merged in;
    returns its kds_final (this rank's share of the groups)."""
    import xpu_b200
    s = xpu_b200.Session(dev, session, kmrels, nrels)
    try:
        for p in parts:
            if p is not None:
                s.merge_final(p)
        final, _ = s.final()
    finally:
        s.close()
    return final


def exchange_final(dev, session: bytes, final, rank, world, kmrels=None, nrels=0, device=None):
    """This rank's share of the job's groups: split, exchange, merge."""
    parts = split_final(dev, session, final, world)
    got = alltoall_bytes(parts, rank, world, device)
    return merge_parts(dev, session, got, kmrels, nrels)

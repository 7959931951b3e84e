"""
Multi-GPU merge of partial-aggregation results by hash partitioning: each
rank splits its groups into one KDS_FORMAT_HASH part per rank by
hash % world on its GPU (xpuB200FinalParts), the parts are exchanged
all-to-all between the GPUs' memories (NCCL over NVLink; a C service would
share the parts buffer by CUDA IPC instead), and each rank merges the parts
it received into a fresh session of the same plan straight from device
memory (xpuB200MergeFinal), so that every group ends on exactly one rank.
alltoall_bytes / merge_parts move host bytes instead (gloo ranks on CPU).
This is the exchange step of a multi-GPU GpuPreAgg whose groups are too
many to gather on one GPU; the reference merges every GPU's kds_final into
the first one instead (__gpuservHandleGpuPreAggFinal,
gpu_service.c:5442-5518).
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


def final_parts(dev, sess_obj, nparts):
    """This session's groups split into nparts hash partitions on its GPU
    (xpuB200FinalParts), back to back in one device buffer from dev.alloc;
    returns (device address, offsets of the nparts parts + the total).
    The caller frees the address."""
    offs = sess_obj.final_parts(nparts)
    base = dev.alloc(max(offs[-1], 256))
    try:
        offs = sess_obj.final_parts(nparts, base, max(offs[-1], 256))
    except Exception:
        dev.free(base)
        raise
    return base, offs


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


def exchange_final(dev, session: bytes, sess_obj, rank, world, kmrels=None, nrels=0, device=None):
    """This rank's share of the job's groups, device to device: the
    session's groups split by hash % world on its GPU (xpuB200FinalParts),
    the parts exchanged between the GPUs' memories in one NCCL
    all_to_all_single (sizes first), and the parts received merged into a
    fresh session straight from device memory (xpuB200MergeFinal on
    device).  No group crosses host memory; the returned kds_final (this
    rank's share) is read back for the caller."""
    import torch
    import torch.distributed as dist
    import xpu_b200
    offs = sess_obj.final_parts(world)
    send = torch.empty(max(offs[-1], 256), dtype=torch.uint8, device=device)
    torch.cuda.synchronize(device)
    offs = sess_obj.final_parts(world, send.data_ptr(), send.numel())
    sizes = [offs[r + 1] - offs[r] for r in range(world)]
    send_n = torch.tensor(sizes, dtype=torch.int64, device=device)
    recv_n = torch.empty(world, dtype=torch.int64, device=device)
    dist.all_to_all_single(recv_n, send_n)
    recv_sizes = recv_n.cpu().tolist()
    recv = torch.empty(max(sum(recv_sizes), 256), dtype=torch.uint8, device=device)
    dist.all_to_all_single(recv[:sum(recv_sizes)], send[:offs[-1]],
                           output_split_sizes=recv_sizes, input_split_sizes=sizes)
    torch.cuda.synchronize(device)
    s = xpu_b200.Session(dev, session, kmrels, nrels)
    try:
        pos = 0
        for n in recv_sizes:
            if n:
                s.merge_final(recv.data_ptr() + pos, on_device=True)
            pos += n
        final, _ = s.final()
    finally:
        s.close()
    return final

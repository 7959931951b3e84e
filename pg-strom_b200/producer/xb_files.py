"""
Chunk producers over files: the counterpart of the reference's relscan.c,
which reads a heap relation's segment files block by block into
KDS_FORMAT_BLOCK chunks (pgstromRelScanChunkDirect, relscan.c:555-742),
and of Arrow_Fdw, which turns the record batches of Arrow IPC files into
KDS_FORMAT_ARROW chunks (arrow_fdw.c:3664-3820).

Dictionary-encoded Arrow columns, which Arrow_Fdw rejects
(arrow_fdw.c:2504), are decoded while the chunk is built: the chunk
carries the plain column (a Utf8 column's offsets and bytes, or the
values), which the executor reads like any other.
"""
import os
import struct

import numpy as np

from xb_producer import BLCKSZ, Column, Table, maxalign

# ArrowType tags of the KDS_FORMAT_ARROW column options (arrow_defs.h)
_TAG_INT, _TAG_FLOAT, _TAG_UTF8, _TAG_BOOL, _TAG_DATE = 2, 3, 5, 6, 8


# ---------------------------------------------------------------- heap files
def write_heap_relation(table: Table, path: str):
    """The table's heap pages as a PostgreSQL relation segment file: 8 KB
    pages in block order, as the storage manager lays them out.  Returns
    the number of blocks."""
    nblocks = 0
    with open(path, "wb") as f:
        for ch in table.block_chunks(pages_per_chunk=8190):
            n, = struct.unpack_from("<I", ch, 16)
            off, = struct.unpack_from("<I", ch, 44)
            f.write(memoryview(ch)[off:off + n * BLCKSZ])
            nblocks += n
    return nblocks


def heap_file_chunks(table_def: Table, path: str, pages_per_chunk=8190, first_blkno=0):
    """KDS_FORMAT_BLOCK chunks of a relation segment file: the column
    layout from table_def (its KDS header), the block numbers, and the
    pages read from the file pages_per_chunk at a time."""
    size = os.path.getsize(path)
    if size % BLCKSZ:
        raise ValueError(f"{path}: {size} bytes is not a whole number of {BLCKSZ}-byte pages")
    nblocks = size // BLCKSZ
    head = table_def.kds_header("b")
    head_len = len(head)
    chunks = []
    with open(path, "rb") as f:
        blk = 0
        while blk < nblocks:
            n = min(pages_per_chunk, nblocks - blk)
            # room for a full chunk's block numbers, as relscan.c sizes it
            block_offset = head_len + maxalign(4 * pages_per_chunk)
            length = block_offset + BLCKSZ * n
            buf = np.zeros(length, dtype=np.uint8)
            buf[:head_len] = np.frombuffer(bytes(head), dtype=np.uint8)
            struct.pack_into("<Q", buf, 0, length)
            struct.pack_into("<I", buf, 16, n)
            struct.pack_into("<II", buf, 44, block_offset, 0)
            buf[head_len:head_len + 4 * n] = np.arange(first_blkno + blk, first_blkno + blk + n,
                                                       dtype=np.uint32).view(np.uint8)
            f.readinto(memoryview(buf)[block_offset:length])
            chunks.append(buf)
            blk += n
    return chunks


IO_PAGE = 4096                  # XPU_B200_IO_PAGE: the file page of an I/O chunk


def heap_file_iovec(table_def: Table, path: str, pages_per_chunk=8190, first_blkno=0, io_pages=None):
    """For reading a relation segment file straight into device memory
    (xpuB200ChunkReadDirect): per chunk, its KDS header with the block
    numbers (base_offset bytes, the part sent from host memory), its
    length, and its I/O vector of (m_offset, fchunk_id, nr_pages) entries
    in IO_PAGE units, as relscan.c builds them (relscan.c:630-663: file
    pages of consecutive blocks merged into one entry)."""
    size = os.path.getsize(path)
    if size % BLCKSZ:
        raise ValueError(f"{path}: {size} bytes is not a whole number of {BLCKSZ}-byte pages")
    nblocks = size // BLCKSZ
    head = bytes(table_def.kds_header("b"))
    head_len = len(head)
    per_block = BLCKSZ // IO_PAGE
    out = []
    blk = 0
    while blk < nblocks:
        n = min(pages_per_chunk, nblocks - blk)
        block_offset = head_len + maxalign(4 * pages_per_chunk)
        length = block_offset + BLCKSZ * n
        hdr = np.zeros(block_offset, dtype=np.uint8)
        hdr[:head_len] = np.frombuffer(head, dtype=np.uint8)
        struct.pack_into("<Q", hdr, 0, length)
        struct.pack_into("<I", hdr, 16, n)
        struct.pack_into("<II", hdr, 44, block_offset, 0)
        hdr[head_len:head_len + 4 * n] = np.arange(first_blkno + blk, first_blkno + blk + n,
                                                   dtype=np.uint32).view(np.uint8)
        total = n * per_block
        step = io_pages or total
        iov = [(IO_PAGE * p, blk * per_block + p, min(step, total - p)) for p in range(0, total, step)]
        out.append({"head": hdr, "base_offset": block_offset, "length": length, "iov": iov})
        blk += n
    return out


# --------------------------------------------------------------- Arrow files
def write_arrow_ipc(path: str, columns: dict, dictionary=(), batch_rows=1 << 20):
    """An Arrow IPC file of the columns (name -> numpy array, or list of
    str for text); columns named in 'dictionary' are dictionary-encoded.
    Date columns are numpy datetime64[D] arrays."""
    import pyarrow as pa
    arrays, names = [], []
    for name, vals in columns.items():
        if isinstance(vals, np.ndarray) and vals.dtype.kind == "M":
            a = pa.array(vals.astype("datetime64[D]"), type=pa.date32())
        elif isinstance(vals, np.ndarray):
            a = pa.array(vals)
        else:
            a = pa.array(vals, type=pa.string())
        if name in dictionary:
            a = a.dictionary_encode()
        arrays.append(a)
        names.append(name)
    tbl = pa.Table.from_arrays(arrays, names=names)
    with pa.OSFile(path, "wb") as sink:
        with pa.ipc.new_file(sink, tbl.schema) as w:
            for batch in tbl.to_batches(max_chunksize=batch_rows):
                w.write_batch(batch)


def _column_type(t):
    import pyarrow as pa
    if pa.types.is_dictionary(t):
        t = t.value_type
    if pa.types.is_int64(t):
        return "int8"
    if pa.types.is_int32(t):
        return "int4"
    if pa.types.is_int16(t):
        return "int2"
    if pa.types.is_boolean(t):
        return "bool"
    if pa.types.is_float64(t):
        return "float8"
    if pa.types.is_date32(t):
        return "date"
    if pa.types.is_string(t):
        return "text"
    raise ValueError(f"Arrow type {t} is not supported by the chunk producer")


def _buffers(arr):
    """the KDS column entry of one Arrow array (dictionary decoded)"""
    import pyarrow as pa
    if pa.types.is_dictionary(arr.type):
        arr = arr.dictionary_decode()
    n = len(arr)
    t = arr.type
    bufs = arr.buffers()
    ent = {}
    if arr.null_count:
        validity = np.frombuffer(bufs[0], dtype=np.uint8)
        off = arr.offset
        if off % 8:
            raise ValueError("sliced Arrow arrays with a bit offset are not supported")
        ent["validity"] = validity[off // 8:off // 8 + (n + 7) // 8].copy()
    if pa.types.is_string(t):
        offs = np.frombuffer(bufs[1], dtype=np.int32)[arr.offset:arr.offset + n + 1]
        data = np.frombuffer(bufs[2], dtype=np.uint8) if bufs[2] is not None else np.zeros(0, np.uint8)
        base = int(offs[0])
        ent.update({"tag": _TAG_UTF8, "values": (offs - base).astype(np.int32),
                    "data": data[base:int(offs[-1])].copy()})
        return ent
    if pa.types.is_boolean(t):
        # bit-packed values, re-based so that row 0 is bit 0
        bits = np.unpackbits(np.frombuffer(bufs[1], dtype=np.uint8), bitorder="little")
        vals = np.packbits(bits[arr.offset:arr.offset + n], bitorder="little")
        ent.update({"tag": _TAG_BOOL, "values": vals})
        return ent
    width = {"int8": 8, "int4": 4, "int2": 2, "float8": 8, "date": 4}[_column_type(t)]
    vals = np.frombuffer(bufs[1], dtype=np.uint8)[arr.offset * width:(arr.offset + n) * width].copy()
    ent["values"] = vals
    if pa.types.is_floating(t):
        ent.update({"tag": _TAG_FLOAT, "precision": 2})
    elif pa.types.is_date32(t):
        ent.update({"tag": _TAG_DATE, "unit": 0})
    else:
        ent.update({"tag": _TAG_INT, "bitwidth": 8 * width})
    return ent


def arrow_ipc_chunks(path: str, columns=None):
    """KDS_FORMAT_ARROW chunks, one per record batch of an Arrow IPC file,
    and the Table describing their columns.  Dictionary columns come out
    decoded.  'columns' names the fields to load, in the order they become
    the chunk's attributes (default: every field); the others are not
    read, as Arrow_Fdw sets up I/O only for the referenced columns of a
    record batch (src/arrow_fdw.c:3750-3768)."""
    import pyarrow as pa
    reader = pa.ipc.open_file(pa.memory_map(path, "r"))
    schema = reader.schema
    names = list(columns) if columns is not None else [f.name for f in schema]
    index = {f.name: j for j, f in enumerate(schema)}
    missing = [n for n in names if n not in index]
    if missing:
        raise ValueError(f"{path}: no field named {', '.join(missing)}")
    cols = [Column(n, _column_type(schema.field(index[n]).type)) for n in names]
    chunks = []
    for i in range(reader.num_record_batches):
        batch = reader.get_batch(i)
        t = Table(os.path.basename(path), cols, batch.num_rows)
        chunks.append(t.arrow_kds({n: _buffers(batch.column(index[n])) for n in names}))
    return chunks, Table(os.path.basename(path), cols, 0)

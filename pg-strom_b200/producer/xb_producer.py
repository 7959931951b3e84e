"""
Seeded chunk and session producer for the B200 executor.

This module plays the part of PG-Strom's host side that lies outside the
executor path: it writes real PostgreSQL heap pages into KDS_FORMAT_BLOCK
chunks (relscan.c:555-742), packs inner relations into KDS_FORMAT_HASH /
kern_multirels buffers (gpu_join.c:2129-2164, :2171-2375), lays out
KDS_FORMAT_ARROW chunks (arrow_fdw.c:3664-3820) and encodes query
expressions as kern_expression bytecode inside a kern_session_info, in the
byte format codegen.c emits (codegen.c:1643-1900, :3149-3700, :3961-4357)
and pgstromBuildSessionInfo packs (executor.c:518-801).

It is test and benchmark infrastructure: the executor under test only ever
sees the byte buffers produced here.
"""
import ctypes
import os
import struct
from dataclasses import dataclass, field

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BLCKSZ = 8192
KVEC_UNITSZ = 1024


def maxalign(x):
    return (x + 7) & ~7


def intalign(x):
    return (x + 3) & ~3


def typealign(a, x):
    return (x + a - 1) & ~(a - 1)


# ---------------------------------------------------------------------------
# opcodes: numeric values of the wire ABI (include/pgstrom_opcodes.h)
# ---------------------------------------------------------------------------
def _load_opcodes():
    path = os.path.join(HERE, "..", "..", "include", "pgstrom_opcodes.h")
    ops = {}
    with open(path) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 3 and parts[0] == "#define" and parts[1].startswith(("FuncOpCode__", "TypeOpCode__")):
                try:
                    ops[parts[1]] = int(parts[2])
                except ValueError:
                    pass
    return ops


OPS = _load_opcodes()


def FOP(name):
    return OPS["FuncOpCode__" + name]


def TOP(name):
    return OPS["TypeOpCode__" + name]


KERN_EXPRESSION_MAGIC = 0x4B657870

# KAGG actions (xpu_common.h:2354-2375)
KAGG = dict(VREF=101, NROWS_ANY=201, NROWS_COND=202, PMIN_INT32=302, PMIN_INT64=303,
            PMIN_FP64=304, PMAX_INT32=402, PMAX_INT64=403, PMAX_FP64=404, PSUM_INT=501,
            PSUM_INT64=502, PSUM_FP=503, PSUM_NUMERIC=504, PAVG_INT=601, PAVG_INT64=602,
            PAVG_FP=603, PAVG_NUMERIC=604, STDDEV=701, COVAR=801)


# ---------------------------------------------------------------------------
# PostgreSQL types
# ---------------------------------------------------------------------------
@dataclass(frozen=True)
class PgType:
    name: str
    oid: int
    attlen: int
    attalign: int
    byval: bool
    kvec_value_sz: int      # bytes per kvec element beyond isnull


PGTYPES = {
    "bool": PgType("bool", 16, 1, 1, True, 1),
    "int2": PgType("int2", 21, 2, 2, True, 2),
    "int4": PgType("int4", 23, 4, 4, True, 4),
    "int8": PgType("int8", 20, 8, 8, True, 8),
    "float8": PgType("float8", 701, 8, 8, True, 8),
    "numeric": PgType("numeric", 1700, -1, 4, False, 1 + 2 + 16 + 8),
    "text": PgType("text", 25, -1, 4, False, 4 + 8),
    "bytea": PgType("bytea", 17, -1, 4, False, 4 + 8),
    "date": PgType("date", 1082, 4, 4, True, 4),
}


def kvec_sizeof(t):
    """Approximate sizeof(kvec_<type>_t): isnull[] plus value arrays."""
    return KVEC_UNITSZ * (1 + PGTYPES[t].kvec_value_sz) + 16


def numeric_typmod(precision, scale):
    return ((precision << 16) | scale) + 4


# ---------------------------------------------------------------------------
# datum encoders
# ---------------------------------------------------------------------------
def encode_varlena(payload: bytes, hdr4=False) -> bytes:
    """PostgreSQL on-disk varlena: 1-byte header when it fits, else (or
    with hdr4) the 4-byte header of an inline uncompressed datum."""
    n = len(payload)
    if n + 1 <= 127 and not hdr4:
        return bytes([((n + 1) << 1) | 1]) + payload
    return struct.pack("<I", (n + 4) << 2) + payload


def encode_numeric(unscaled: int, scale: int, long_fmt=False, hdr4=False) -> bytes:
    """numeric value unscaled * 10^-scale in PostgreSQL's short (or long)
    on-disk format: base-10000 digits, weight of the first digit, dscale.
    long_fmt writes the NUMERIC_LONG header (n_sign_dscale, n_weight) that
    PostgreSQL uses when dscale or weight do not fit the short header (and
    wrote for every value before 9.1); hdr4 gives the datum a 4-byte
    varlena header."""
    neg = unscaled < 0
    v = -unscaled if neg else unscaled
    # decimal digits aligned so that the fractional part fills whole groups
    frac_groups = (scale + 3) // 4
    pad = frac_groups * 4 - scale
    v_aligned = v * (10 ** pad)
    digits = []
    while v_aligned > 0:
        digits.append(v_aligned % 10000)
        v_aligned //= 10000
    digits.reverse()
    if not digits:
        weight = 0
    else:
        weight = len(digits) - frac_groups - 1
    # strip leading zero groups (cannot happen) and trailing zero groups
    while digits and digits[-1] == 0:
        digits.pop()
    while digits and digits[0] == 0:
        digits.pop(0)
        weight -= 1
    if not digits:
        weight = 0
        neg = False
    if scale <= 0x3F and -64 <= weight <= 63 and not long_fmt:
        head = 0x8000 | (0x2000 if neg else 0) | (scale << 7) | (weight & 0x7F)
        body = struct.pack("<H", head) + b"".join(struct.pack("<h", d) for d in digits)
    else:
        head = (0x4000 if neg else 0) | (scale & 0x3FFF)
        body = struct.pack("<Hh", head, weight) + b"".join(struct.pack("<h", d) for d in digits)
    return encode_varlena(body, hdr4)


def encode_varlena_list(images):
    """List of encoded datums (bytes) -> (blob, offsets)."""
    offs = np.zeros(len(images) + 1, dtype=np.int64)
    np.cumsum([len(p) for p in images], out=offs[1:])
    return np.frombuffer(b"".join(images), dtype=np.uint8).copy(), offs


def encode_numeric_array(unscaled: np.ndarray, scale: int):
    """Vectorised encode_numeric for |value| < 10^8 with scale <= 4.
    Returns (blob uint8, offsets int64[n+1])."""
    assert 0 <= scale <= 4
    v = unscaled.astype(np.int64)
    neg = v < 0
    a = np.abs(v) * (10 ** (4 - scale)) if scale > 0 else np.abs(v)
    if scale > 0:
        frac = a % 10000
        ip = a // 10000
    else:
        frac = np.zeros_like(a)
        ip = a
    assert int(ip.max(initial=0)) < 10 ** 8
    ip_hi = ip // 10000
    ip_lo = ip % 10000
    # digit groups: [ip_hi, ip_lo, frac] for scale > 0, [ip_hi, ip_lo] otherwise
    if scale > 0:
        groups = np.stack([ip_hi, ip_lo, frac], axis=1)
        base_weight = 1                          # weight of ip_hi
    else:
        groups = np.stack([ip_hi, ip_lo], axis=1)
        base_weight = 1
    ng = groups.shape[1]
    nz = groups != 0
    any_nz = nz.any(axis=1)
    first = np.where(any_nz, nz.argmax(axis=1), 0)
    last = np.where(any_nz, ng - 1 - nz[:, ::-1].argmax(axis=1), -1)
    ndig = np.where(any_nz, last - first + 1, 0)
    weight = np.where(any_nz, base_weight - first, 0)
    negf = neg & any_nz
    head = (0x8000 | (negf.astype(np.int64) << 13) | (scale << 7) | (weight & 0x7F)).astype(np.uint16)
    sizes = 1 + 2 + 2 * ndig                     # 1B varlena header
    offs = np.zeros(len(v) + 1, dtype=np.int64)
    np.cumsum(sizes, out=offs[1:])
    blob = np.zeros(int(offs[-1]), dtype=np.uint8)
    starts = offs[:-1]
    blob[starts] = ((sizes << 1) | 1).astype(np.uint8)
    blob[starts + 1] = (head & 0xFF).astype(np.uint8)
    blob[starts + 2] = (head >> 8).astype(np.uint8)
    for k in range(ng):
        use = ndig > k
        g = groups[np.arange(len(v)), np.clip(first + k, 0, ng - 1)]
        pos = starts + 3 + 2 * k
        blob[pos[use]] = (g[use] & 0xFF).astype(np.uint8)
        blob[pos[use] + 1] = ((g[use] >> 8) & 0xFF).astype(np.uint8)
    return blob, offs


def encode_text_array(strings):
    """List of str/bytes -> (blob, offsets) of short varlenas."""
    parts = [encode_varlena(s.encode() if isinstance(s, str) else s) for s in strings]
    offs = np.zeros(len(parts) + 1, dtype=np.int64)
    np.cumsum([len(p) for p in parts], out=offs[1:])
    return np.frombuffer(b"".join(parts), dtype=np.uint8).copy(), offs


def encode_text_from_dict(codes: np.ndarray, dictionary):
    """Dictionary codes -> varlena blob (vectorised via per-code images)."""
    imgs = [encode_varlena(s.encode()) for s in dictionary]
    lens = np.array([len(x) for x in imgs], dtype=np.int64)
    sizes = lens[codes]
    offs = np.zeros(len(codes) + 1, dtype=np.int64)
    np.cumsum(sizes, out=offs[1:])
    blob = np.zeros(int(offs[-1]), dtype=np.uint8)
    maxl = int(lens.max())
    table = np.zeros((len(imgs), maxl), dtype=np.uint8)
    for i, x in enumerate(imgs):
        table[i, :len(x)] = np.frombuffer(x, dtype=np.uint8)
    for k in range(maxl):
        use = sizes > k
        blob[offs[:-1][use] + k] = table[codes[use], k]
    return blob, offs


# ---------------------------------------------------------------------------
# host hash (hash_any / pg_hash_merge), as gpu_join.c:1549-1584 computes it
# ---------------------------------------------------------------------------
def _rot(x, k):
    return ((x << k) | (x >> (32 - k))) & 0xFFFFFFFF


def hash_any(data: bytes) -> int:
    """Bob Jenkins' lookup3 hashlittle() as used by PostgreSQL hash_any()."""
    M = 0xFFFFFFFF
    n = len(data)
    a = b = c = (0x9E3779B9 + n + 3923095) & M
    k = 0
    while n >= 12:
        a = (a + int.from_bytes(data[k:k + 4], "little")) & M
        b = (b + int.from_bytes(data[k + 4:k + 8], "little")) & M
        c = (c + int.from_bytes(data[k + 8:k + 12], "little")) & M
        a = (a - c) & M; a ^= _rot(c, 4); c = (c + b) & M
        b = (b - a) & M; b ^= _rot(a, 6); a = (a + c) & M
        c = (c - b) & M; c ^= _rot(b, 8); b = (b + a) & M
        a = (a - c) & M; a ^= _rot(c, 16); c = (c + b) & M
        b = (b - a) & M; b ^= _rot(a, 19); a = (a + c) & M
        c = (c - b) & M; c ^= _rot(b, 4); b = (b + a) & M
        k += 12
        n -= 12
    tail = data[k:]
    if n > 8:
        c = (c + (int.from_bytes(tail[8:], "little") << 8)) & M
        b = (b + int.from_bytes(tail[4:8], "little")) & M
        a = (a + int.from_bytes(tail[0:4], "little")) & M
    elif n > 4:
        b = (b + int.from_bytes(tail[4:], "little")) & M
        a = (a + int.from_bytes(tail[0:4], "little")) & M
    elif n > 0:
        a = (a + int.from_bytes(tail, "little")) & M
    c ^= b; c = (c - _rot(b, 14)) & M
    a ^= c; a = (a - _rot(c, 11)) & M
    b ^= a; b = (b - _rot(a, 25)) & M
    c ^= b; c = (c - _rot(b, 16)) & M
    a ^= c; a = (a - _rot(c, 4)) & M
    b ^= a; b = (b - _rot(a, 14)) & M
    c ^= b; c = (c - _rot(b, 24)) & M
    return c


def hash_u32_array(v: np.ndarray, nbytes: int) -> np.ndarray:
    """Vectorised hash_any() of 1/2/4-byte little-endian integers."""
    M = np.uint64(0xFFFFFFFF)
    v = v.astype(np.int64).astype(np.uint64) & np.uint64((1 << (8 * nbytes)) - 1)
    init = np.uint64((0x9E3779B9 + nbytes + 3923095) & 0xFFFFFFFF)
    a = (init + v) & M
    b = np.full_like(a, init)
    c = np.full_like(a, init)
    return _final_vec(a, b, c)


def hash_u64_array(v: np.ndarray) -> np.ndarray:
    M = np.uint64(0xFFFFFFFF)
    u = v.astype(np.int64).view(np.uint64) if v.dtype != np.uint64 else v
    init = np.uint64((0x9E3779B9 + 8 + 3923095) & 0xFFFFFFFF)
    a = (init + (u & M)) & M
    b = (init + (u >> np.uint64(32))) & M
    c = np.full_like(a, init)
    return _final_vec(a, b, c)


def _final_vec(a, b, c):
    M = np.uint64(0xFFFFFFFF)

    def rot(x, k):
        return ((x << np.uint64(k)) | (x >> np.uint64(32 - k))) & M
    c = (c ^ b); c = (c - rot(b, 14)) & M
    a = (a ^ c); a = (a - rot(c, 11)) & M
    b = (b ^ a); b = (b - rot(a, 25)) & M
    c = (c ^ b); c = (c - rot(b, 16)) & M
    a = (a ^ c); a = (a - rot(c, 4)) & M
    b = (b ^ a); b = (b - rot(a, 14)) & M
    c = (c ^ b); c = (c - rot(b, 24)) & M
    return c.astype(np.uint32)


def hash_merge_array(prev: np.ndarray, nxt: np.ndarray) -> np.ndarray:
    p = prev.astype(np.uint32)
    return (((p >> np.uint32(3)) | (p << np.uint32(29))) ^ nxt.astype(np.uint32)).astype(np.uint32)


# ---------------------------------------------------------------------------
# tables and chunk builders
# ---------------------------------------------------------------------------
_HG = None


def _heapgen():
    global _HG
    if _HG is None:
        so = os.path.join(HERE, "libxb_heapgen.so")
        src = os.path.join(HERE, "xb_heapgen.c")
        if not os.path.exists(so) or os.path.getmtime(so) < os.path.getmtime(src):
            rc = os.system(f"gcc -O2 -fPIC -shared -o {so} {src}")
            if rc != 0:
                raise RuntimeError("failed to build libxb_heapgen.so")
        _HG = ctypes.CDLL(so)
        _HG.hg_build_pages.restype = ctypes.c_int64
        _HG.hg_build_hash_kds.restype = ctypes.c_int64
        _HG.hg_minimal_tuple_len.restype = ctypes.c_int64
    return _HG


class _HgCol(ctypes.Structure):
    _fields_ = [("attlen", ctypes.c_int32), ("attalign", ctypes.c_int32)]


@dataclass
class Column:
    name: str
    typ: str
    typmod: int = -1
    values: object = None       # fixed: np.ndarray; varlena: (blob, offsets)
    nulls: object = None        # np.ndarray[bool] or None


@dataclass
class Table:
    name: str
    columns: list
    nrows: int
    table_oid: int = 16384

    def col(self, name):
        for c in self.columns:
            if c.name == name:
                return c
        raise KeyError(name)

    def resno(self, name):
        for i, c in enumerate(self.columns):
            if c.name == name:
                return i + 1
        raise KeyError(name)

    # -- ctypes argument arrays for the C helper --
    def _c_args(self):
        n = len(self.columns)
        cols = (_HgCol * n)()
        data = (ctypes.c_void_p * n)()
        voffs = (ctypes.c_void_p * n)()
        nulls = (ctypes.c_void_p * n)()
        keep = []
        for j, c in enumerate(self.columns):
            t = PGTYPES[c.typ]
            cols[j].attlen = t.attlen
            cols[j].attalign = t.attalign
            if t.attlen > 0:
                arr = np.ascontiguousarray(c.values)
                assert arr.dtype.itemsize == t.attlen, (c.name, arr.dtype)
                keep.append(arr)
                data[j] = arr.ctypes.data
                voffs[j] = None
            else:
                blob, offs = c.values
                blob = np.ascontiguousarray(blob, dtype=np.uint8)
                offs = np.ascontiguousarray(offs, dtype=np.int64)
                keep += [blob, offs]
                data[j] = blob.ctypes.data
                voffs[j] = offs.ctypes.data
            if c.nulls is not None:
                nm = np.ascontiguousarray(c.nulls, dtype=np.uint8)
                keep.append(nm)
                nulls[j] = nm.ctypes.data
            else:
                nulls[j] = None
        return cols, data, voffs, nulls, keep

    def kds_header(self, fmt: str, nitems: int = 0) -> bytearray:
        """kern_data_store header + colmeta[] (relscan.c:179-345)."""
        ncols = len(self.columns)
        head_len = maxalign(72 + 168 * ncols)
        buf = bytearray(head_len)
        struct.pack_into("<QQIIc??xIiI", buf, 0, 0, 0, nitems, ncols, fmt.encode(),
                         any(PGTYPES[c.typ].attlen < 0 for c in self.columns), False,
                         0, -1, self.table_oid)
        struct.pack_into("<I", buf, 68, ncols)                  # nr_colmeta
        attcacheoff = 0 if fmt in ("r", "h", "b") else -1
        for j, c in enumerate(self.columns):
            t = PGTYPES[c.typ]
            off = 72 + 168 * j
            if attcacheoff < 0:
                cache = -1
            elif t.attlen > 0:
                cache = typealign(t.attalign, attcacheoff)
                attcacheoff = cache + t.attlen
            else:
                a = typealign(t.attalign, attcacheoff)
                cache = a if a == attcacheoff else -1
                attcacheoff = -1
            struct.pack_into("<?bhhhIibchI", buf, off, t.byval, t.attalign, t.attlen, j + 1, cache,
                             t.oid, c.typmod, ord("b"), fmt.encode(), 0, off)
            buf[off + 28:off + 28 + len(c.name.encode())] = c.name.encode()
            struct.pack_into("<q", buf, off + 112, -0)          # virtual_offset = 0
        return buf

    def block_chunks(self, pages_per_chunk=8190, first_blkno=0):
        """KDS_FORMAT_BLOCK chunks (list of bytes-like np.uint8 arrays)."""
        hg = _heapgen()
        cols, data, voffs, nulls, keep = self._c_args()
        chunks = []
        row = 0
        blk = first_blkno
        head = self.kds_header("b")
        head_len = len(head)
        while row < self.nrows:
            block_offset = head_len + maxalign(4 * pages_per_chunk)
            buf = np.zeros(block_offset + BLCKSZ * pages_per_chunk, dtype=np.uint8)
            nxt = ctypes.c_int64(0)
            np_ = hg.hg_build_pages(len(self.columns), cols, data, voffs, nulls,
                                    ctypes.c_int64(row), ctypes.c_int64(self.nrows),
                                    ctypes.c_void_p(buf.ctypes.data + block_offset),
                                    ctypes.c_int64(pages_per_chunk), ctypes.c_uint32(blk),
                                    ctypes.c_uint32(2), ctypes.byref(nxt))
            if np_ <= 0:
                raise RuntimeError("heap page build failed")
            length = block_offset + BLCKSZ * np_
            buf = buf[:length]
            buf[:head_len] = np.frombuffer(bytes(head), dtype=np.uint8)
            struct.pack_into("<Q", buf, 0, length)
            struct.pack_into("<I", buf, 16, np_)                 # nitems (blocks)
            struct.pack_into("<II", buf, 44, block_offset, 0)    # block_offset, block_nloaded
            blknums = np.arange(blk, blk + np_, dtype=np.uint32)
            buf[head_len:head_len + 4 * np_] = blknums.view(np.uint8)
            chunks.append(buf)
            row = nxt.value
            blk += np_
        return chunks

    def row_chunks(self, rows_per_chunk=20_000):
        """KDS_FORMAT_ROW chunks of the table's rows in table order, the
        outer-chunk form the reference's __gpuscan_load_source_row reads
        (cuda_gpuscan.cu:646-700): the header, the row index of nitems
        offsets counted back from the chunk's end (KDS_GET_TUPITEM,
        xpu_common.h:1337-1345), and the rows as kern_tupitems from the end,
        8-byte aligned.  A kern_tupitem is its length and hash words, no
        transaction attributes, the heap tuple's header from t_infomask2 on
        with t_hoff kept relative to the heap tuple (MINIMAL_TUPLE_OFFSET
        bytes before the item), its data, and the row id at its tail."""
        images = []
        for ch in self.block_chunks():
            nblocks, = struct.unpack_from("<I", ch, 16)
            block_offset, = struct.unpack_from("<I", ch, 44)
            for b in range(nblocks):
                base = block_offset + b * BLCKSZ
                lower, = struct.unpack_from("<H", ch, base + 12)
                for i in range((lower - 24) // 4):
                    lp, = struct.unpack_from("<I", ch, base + 24 + 4 * i)
                    off, flags, ln = lp & 0x7fff, (lp >> 15) & 3, lp >> 17
                    if flags != 1:
                        continue
                    images.append(bytes(ch[base + off + 18:base + off + ln]))
        chunks = []
        for c0 in range(0, len(images), rows_per_chunk):
            part = images[c0:c0 + rows_per_chunk]
            head = self.kds_header("r", len(part))
            head_len = len(head)
            items = []
            for rowid, tail in enumerate(part):
                t_len = 10 + len(tail) + 4
                items.append(struct.pack("<IIBB", t_len, 0, 0, 0) + tail + struct.pack("<I", rowid))
            sizes = [maxalign(len(t)) for t in items]
            usage = sum(sizes)
            length = head_len + 8 * len(part) + usage
            buf = np.zeros(length, dtype=np.uint8)
            buf[:head_len] = np.frombuffer(bytes(head), dtype=np.uint8)
            struct.pack_into("<QQ", buf, 0, length, usage)
            back = 0
            for j, (t, sz) in enumerate(zip(items, sizes)):
                back += sz
                struct.pack_into("<Q", buf, head_len + 8 * j, back)
                buf[length - back:length - back + len(t)] = np.frombuffer(t, dtype=np.uint8)
            chunks.append(buf)
        return chunks

    def hash_kds(self, hashes: np.ndarray) -> np.ndarray:
        """KDS_FORMAT_HASH inner buffer with host-computed hash per row."""
        hg = _heapgen()
        cols, data, voffs, nulls, keep = self._c_args()
        head = self.kds_header("h", self.nrows)
        head_len = len(head)
        nslots = 20000 if self.nrows <= 5000 else (20000 + 2 * self.nrows if self.nrows <= 4000000
                                                   else 8020000 + self.nrows)
        est = head_len + 8 * (nslots + self.nrows)
        lens = self._minimal_lens_vec()
        usage = int(np.sum((8 + lens + 4 + 7) // 8 * 8))
        length = est + usage
        buf = np.zeros(length, dtype=np.uint8)
        buf[:head_len] = np.frombuffer(bytes(head), dtype=np.uint8)
        struct.pack_into("<QQ", buf, 0, length, usage)
        struct.pack_into("<I", buf, 40, nslots)                  # hash_nslots
        hashes = np.ascontiguousarray(hashes, dtype=np.uint32)
        got = hg.hg_build_hash_kds(len(self.columns), cols, data, voffs, nulls,
                                   ctypes.c_int64(self.nrows), ctypes.c_void_p(hashes.ctypes.data),
                                   ctypes.c_void_p(buf.ctypes.data), ctypes.c_int64(head_len),
                                   ctypes.c_uint32(nslots), ctypes.c_int64(length))
        if got != usage:
            raise RuntimeError(f"hash kds build mismatch {got} != {usage}")
        return buf

    def _minimal_lens_vec(self):
        """t_len of every row's MinimalTuple, vectorised (fixed or varlena)."""
        n = self.nrows
        hasnull = np.zeros(n, dtype=bool)
        for c in self.columns:
            if c.nulls is not None:
                hasnull |= c.nulls.astype(bool)
        hoff = np.where(hasnull, maxalign(23 + (len(self.columns) + 7) // 8), 24)
        off = np.zeros(n, dtype=np.int64)
        for c in self.columns:
            t = PGTYPES[c.typ]
            isn = c.nulls.astype(bool) if c.nulls is not None else np.zeros(n, dtype=bool)
            if t.attlen > 0:
                new = ((off + t.attalign - 1) // t.attalign) * t.attalign + t.attlen
            else:
                blob, offs = c.values
                first = blob[offs[:-1]]
                l = np.diff(offs)
                aligned = ((off + t.attalign - 1) // t.attalign) * t.attalign
                new = np.where((first & 1) == 1, off, aligned) + l
            off = np.where(isn, off, new)
        return hoff - 8 + off

    def arrow_kds(self, arrow_cols: dict) -> np.ndarray:
        """KDS_FORMAT_ARROW chunk.  arrow_cols maps column name to a dict with
        Arrow buffers: {'tag', 'bitwidth'/'precision'/'unit', 'validity',
        'values', 'offsets', 'data'}."""
        ncols = len(self.columns)
        head = self.kds_header("a", self.nrows)
        head_len = len(head)
        bufs = []
        pos = (head_len + 63) & ~63
        layout = []
        for c in self.columns:
            ac = arrow_cols[c.name]
            ent = {}
            for key in ("validity", "values", "data"):
                b = ac.get(key)
                if b is None:
                    ent[key] = (0, 0)
                    continue
                b = np.ascontiguousarray(b).view(np.uint8).ravel()
                ent[key] = (pos, len(b))
                bufs.append((pos, b))
                pos = (pos + len(b) + 63) & ~63
            layout.append(ent)
        length = pos
        buf = np.zeros(length, dtype=np.uint8)
        buf[:head_len] = np.frombuffer(bytes(head), dtype=np.uint8)
        struct.pack_into("<QQ", buf, 0, length, length)
        for p, b in bufs:
            buf[p:p + len(b)] = b
        for j, (c, ent) in enumerate(zip(self.columns, layout)):
            ac = arrow_cols[c.name]
            off = 72 + 168 * j
            struct.pack_into("<h", buf, off + 6, -1)             # attcacheoff
            # ArrowTypeOptions at +92: tag, unitsz, align, union
            tag = ac["tag"]
            struct.pack_into("<ihH", buf, off + 92, tag, ac.get("unitsz", 0), ac.get("align", 0))
            if tag == 2:       # Int
                struct.pack_into("<HB", buf, off + 100, ac["bitwidth"], 1)
            elif tag == 3:     # FloatingPoint
                struct.pack_into("<i", buf, off + 100, ac["precision"])
            elif tag == 8:     # Date
                struct.pack_into("<i", buf, off + 100, ac.get("unit", 0))
            struct.pack_into("<i", buf, off + 108, j)            # field_index
            struct.pack_into("<q", buf, off + 112, 0)            # virtual_offset
            nm, vl, ex = ent["validity"], ent["values"], ent["data"]
            struct.pack_into("<QQQQQQ", buf, off + 120, nm[0], nm[1], vl[0], vl[1], ex[0], ex[1])
        return buf


def kern_multirels(inner_kds_list) -> np.ndarray:
    """kern_multirels with the inner KDS_FORMAT_HASH buffers appended."""
    n = len(inner_kds_list)
    head = maxalign(32 + 56 * n)
    pos = head
    offs = []
    for k in inner_kds_list:
        offs.append(pos)
        pos = maxalign(pos + len(k))
    buf = np.zeros(pos, dtype=np.uint8)
    struct.pack_into("<QQQI", buf, 0, pos, 0, 0, n)
    for i, (k, o) in enumerate(zip(inner_kds_list, offs)):
        base = 32 + 56 * i
        struct.pack_into("<QQQQQh????xxQ", buf, base, 0, 0, o, 0, 0, 0, False, False, False, False, 0)
        buf[o:o + len(k)] = k
    return buf


# ---------------------------------------------------------------------------
# expressions and bytecode (codegen.c restated for the shapes used here)
# ---------------------------------------------------------------------------
class Expr:
    pass


@dataclass
class Var(Expr):
    depth: int
    resno: int
    typ: str
    typmod: int = -1


@dataclass
class Const(Expr):
    typ: str
    value: object           # python value; None = NULL


@dataclass
class Param(Expr):
    typ: str
    value: object


@dataclass
class Func(Expr):
    op: str                 # FuncOpCode name, e.g. 'int4lt'
    args: list
    typ: str


@dataclass
class BoolOp(Expr):
    kind: str               # 'And' | 'Or' | 'Not'
    args: list
    typ: str = "bool"


@dataclass
class NullTest(Expr):
    arg: Expr
    isnull: bool
    typ: str = "bool"


@dataclass
class Agg:
    action: str             # KAGG action name
    arg: Expr = None
    typmod: int = -1
    arg1: Expr = None       # COVAR's second argument (Y)


def const_image(typ, value):
    t = PGTYPES[typ]
    if typ == "bool":
        return struct.pack("<?", bool(value))
    if typ == "int2":
        return struct.pack("<h", value)
    if typ in ("int4", "date"):
        return struct.pack("<i", value)
    if typ == "int8":
        return struct.pack("<q", value)
    if typ == "float8":
        return struct.pack("<d", value)
    if typ in ("text", "bytea"):
        v = value.encode() if isinstance(value, str) else value
        return struct.pack("<I", (len(v) + 4) << 2) + v
    if typ == "numeric":
        unscaled, scale = value
        return encode_numeric(unscaled, scale)
    raise ValueError(typ)


class _Buf:
    def __init__(self):
        self.b = bytearray()

    def append_aligned(self, data):
        pad = maxalign(len(self.b)) - len(self.b)
        self.b += b"\0" * pad
        pos = len(self.b)
        self.b += data
        return pos

    def finish_kexp(self, head_pos):
        pad = intalign(len(self.b)) - len(self.b)
        self.b += b"\0" * pad
        exptype, opcode = struct.unpack_from("<i", self.b, head_pos + 4)[0], \
            struct.unpack_from("<i", self.b, head_pos + 20)[0]
        magic = (KERN_EXPRESSION_MAGIC ^ ((exptype & 0xFFFFFFFF) << 6) ^ ((opcode & 0xFFFFFFFF) << 14)) & 0xFFFFFFFF
        self.b += struct.pack("<I", magic)
        struct.pack_into("<I", self.b, head_pos, len(self.b) - head_pos)


KSORT = dict(VREF=0, PMINMAX_INT64=1, PMINMAX_FP64=2, PSUM_INT64=3, PSUM_FP64=4, PSUM_NUMERIC=5,
             PAVG_INT64=6, PAVG_FP64=7, PAVG_NUMERIC=8, PVARIANCE_SAMP=9, PVARIANCE_POP=10,
             PCOVAR_CORR=11, PCOVAR_SAMP=12, PCOVAR_POP=13, PCOVAR_AVGX=14, PCOVAR_AVGY=15,
             PCOVAR_COUNT=16, NITEMS=23)


def build_sort_keys(keys, window=None):
    """SortKeys kexp (xpu_common.h:2676-2684): keys = list of (kind name,
    kds_final attribute number, ascending, nulls first); window = (function
    'n' / 'r' / 'd', partition keys, order keys, rank limit) or None."""
    wf, pb, ob, lim = window if window else ("\0", 0, 0, 0)
    body = struct.pack("<i?cxxIHH", len(keys), True, wf.encode(), lim, pb, ob)
    for kind, anum, asc, nf in keys:
        body += struct.pack("<HbbHHixxxxQ", KSORT[kind], 1 if nf else 0, 1 if asc else 0, anum, 0, 0, 0)
    buf = _Buf()
    buf.b += _kexp_head(TOP("int4"), FOP("SortKeys"), 0, 0) + body
    buf.finish_kexp(0)
    return bytes(buf.b)


def _kexp_head(exptype, opcode, nr_args=0, args_offset=0, flags=0):
    return struct.pack("<IiQIiQII", 0, exptype, 0, flags, opcode, 0, nr_args, args_offset)


@dataclass
class KvDef:
    slot: int
    depth: int
    resno: int
    typ: str
    typmod: int
    offset: int             # kvec offset, -1 if none
    maxref: int
    expr: object = None


class SessionBuilder:
    """Builds a kern_session_info blob for a scan/join/pre-agg query."""

    def __init__(self, num_inner_rels=0, task_flags=0x40000001):
        self.nrels = num_inner_rels
        self.kvdefs = []
        self.kvecs_usage = 0
        self.flags = task_flags
        self.params = []

    # -- kvars --
    def _lookup_var(self, v: Var, curr_depth):
        for d in self.kvdefs:
            if d.depth == v.depth and d.resno == v.resno and d.expr is None:
                d.maxref = max(d.maxref, curr_depth)
                return d
        d = KvDef(len(self.kvdefs), v.depth, v.resno, v.typ, v.typmod, self.kvecs_usage, curr_depth)
        self.kvecs_usage += typealign(16, kvec_sizeof(v.typ))
        self.kvdefs.append(d)
        return d

    def _temp(self, expr: Expr, depth):
        for d in self.kvdefs:
            if d.expr is not None and d.expr == expr:
                return d
        d = KvDef(len(self.kvdefs), depth, 0, expr.typ, -1, -1, depth, expr)
        self.kvdefs.append(d)
        return d

    # -- expression encoding --
    def emit(self, buf: _Buf, e: Expr, depth: int, flags=0):
        if isinstance(e, Var):
            d = self._lookup_var(e, depth)
            off = d.offset if (d.offset >= 0 and d.depth != depth) else -1
            pos = buf.append_aligned(_kexp_head(TOP(e.typ), FOP("VarExpr"), flags=flags) +
                                     struct.pack("<iH", off, d.slot))
            buf.finish_kexp(pos)
        elif isinstance(e, Const):
            img = b"" if e.value is None else const_image(e.typ, e.value)
            pos = buf.append_aligned(_kexp_head(TOP(e.typ), FOP("ConstExpr"), flags=flags) +
                                     struct.pack("<I?xxx", PGTYPES[e.typ].oid, e.value is None) + img)
            buf.finish_kexp(pos)
        elif isinstance(e, Param):
            pid = len(self.params)
            self.params.append(None if e.value is None else const_image(e.typ, e.value))
            pos = buf.append_aligned(_kexp_head(TOP(e.typ), FOP("ParamExpr"), flags=flags) +
                                     struct.pack("<I", pid))
            buf.finish_kexp(pos)
        elif isinstance(e, Func):
            pos = buf.append_aligned(_kexp_head(TOP(e.typ), FOP(e.op), len(e.args), 40, flags))
            for a in e.args:
                self.emit(buf, a, depth, flags)
            buf.finish_kexp(pos)
        elif isinstance(e, BoolOp):
            op = {"And": "BoolExpr_And", "Or": "BoolExpr_Or", "Not": "BoolExpr_Not"}[e.kind]
            pos = buf.append_aligned(_kexp_head(TOP("bool"), FOP(op), len(e.args), 40, flags))
            for a in e.args:
                self.emit(buf, a, depth, flags)
            buf.finish_kexp(pos)
        elif isinstance(e, NullTest):
            op = "NullTestExpr_IsNull" if e.isnull else "NullTestExpr_IsNotNull"
            pos = buf.append_aligned(_kexp_head(TOP("bool"), FOP(op), 1, 40, flags))
            self.emit(buf, e.arg, depth, flags)
            buf.finish_kexp(pos)
        else:
            raise TypeError(e)

    def emit_save(self, buf: _Buf, e: Expr, depth: int):
        """SaveExpr(e) into a kvars slot (__try_inject_temporary_expression)."""
        if isinstance(e, Var):
            d = self._lookup_var(e, depth)
        else:
            d = self._temp(e, depth)
        pos = buf.append_aligned(_kexp_head(TOP(e.typ), FOP("SaveExpr"), 1, 48) +
                                 struct.pack("<H", d.slot))
        self.emit(buf, e, depth)
        buf.finish_kexp(pos)
        return d

    def build_expr(self, e: Expr, depth: int) -> bytes:
        buf = _Buf()
        self.emit(buf, e, depth)
        return bytes(buf.b)

    def build_hash_value(self, keys, depth) -> bytes:
        buf = _Buf()
        buf.b += _kexp_head(TOP("int4"), FOP("HashValue"), len(keys), 40)
        for k in keys:
            self.emit(buf, k, depth)
        buf.finish_kexp(0)
        return bytes(buf.b)

    def build_join_quals(self, quals, other_quals, depth) -> bytes:
        buf = _Buf()
        buf.b += _kexp_head(TOP("bool"), FOP("JoinQuals"), len(quals) + len(other_quals), 40)
        for q in quals:
            self.emit(buf, q, depth)
        for q in other_quals:
            self.emit(buf, q, depth, flags=1)
        buf.finish_kexp(0)
        return bytes(buf.b)

    @staticmethod
    def packed(subs: dict, npacked: int, nslots_off: int) -> bytes:
        """Packed expression: subs maps depth -> kexp bytes."""
        sz = maxalign(44 + 4 * nslots_off)
        buf = _Buf()
        buf.b += bytearray(sz)
        offsets = [0] * nslots_off
        n = 0
        for depth in sorted(subs):
            offsets[depth] = buf.append_aligned(subs[depth])
            n += 1
        head = _kexp_head(TOP("int4"), FOP("Packed"), n, sz) + struct.pack("<I", npacked) + \
            struct.pack("<%dI" % nslots_off, *offsets)
        buf.b[:len(head)] = head
        buf.finish_kexp(0)
        return bytes(buf.b)

    def build_loadvars(self, depth) -> bytes:
        items = sorted([(d.resno, d.slot) for d in self.kvdefs if d.depth == depth and d.expr is None])
        if not items:
            return None
        args_off = maxalign(48 + 4 * len(items))
        body = _kexp_head(TOP("int4"), FOP("LoadVars"), 0, args_off) + struct.pack("<ii", depth, len(items))
        body += b"".join(struct.pack("<hh", r, s) for r, s in items)
        buf = _Buf()
        buf.b += body + b"\0" * (args_off - len(body))
        buf.finish_kexp(0)
        return bytes(buf.b)

    def build_movevars(self, depth) -> bytes:
        items = [d for d in self.kvdefs if d.offset >= 0 and 0 <= d.depth <= depth and d.maxref > depth]
        if not items:
            return None
        sz = maxalign(48 + 8 * len(self.kvdefs))
        body = _kexp_head(TOP("int4"), FOP("MoveVars"), 0, sz) + struct.pack("<ii", depth, len(items))
        body += b"".join(struct.pack("<ih?x", d.offset, d.slot, d.depth == depth) for d in items)
        buf = _Buf()
        buf.b += body + b"\0" * (sz - len(body))
        buf.finish_kexp(0)
        return bytes(buf.b)

    # -- the whole session --
    def build_projection(self, tlist, depth, hash_keys=None):
        """Projection kexp (codegen_build_projection, codegen.c:3880-3950):
        one SaveExpr per target entry into a kvars slot, skipped when an
        earlier entry already saved into the same slot
        (try_inject_projection_expression, codegen.c:3412-3437);
        u.proj.slot_id[] names each output attribute's slot.  hash_keys
        (rows for a pinned inner buffer) appends a HashValue over them,
        found at u.proj.hash (codegen.c:3933-3941)."""
        nattrs = len(tlist)
        head_sz = maxalign(48 + 2 * nattrs)
        buf = _Buf()
        buf.b += bytearray(head_sz)
        slots, nargs = [], 0
        for e in tlist:
            pos = len(buf.b)
            d = self.emit_save(buf, e, depth)
            if d.slot in slots:
                del buf.b[pos:]
            else:
                nargs += 1
            slots.append(d.slot)
        hash_off = 0
        if hash_keys:
            hash_off = buf.append_aligned(self.build_hash_value(hash_keys, depth))
        head = _kexp_head(TOP("int4"), FOP("Projection"), nargs, head_sz) + \
            struct.pack("<Ii", hash_off, nattrs) + struct.pack("<%dH" % nattrs, *slots)
        buf.b[:len(head)] = head
        buf.finish_kexp(0)
        return bytes(buf.b)

    def build(self, *, scan_quals=None, joins=(), groupby_keys=(), aggs=(),
              ngroups_estimate=100.0, final_tlist=None, projection=None,
              htup_margin=0, projection_hash=None, proj_nslots=0, sort_keys=None,
              sort_window=None, sort_limit=0, join_inner_handle=0) -> bytes:
        """joins: list of (outer_hash_keys, join_quals, other_quals) for
        depth 1..n.  groupby_keys: list of Expr; aggs: list of Agg.  The
        partial-aggregation target list is aggs then keys (gpu_preagg.c:
        2080-2097).  projection: list of Expr written as KDS_FORMAT_ROW rows
        (a scan/join without GROUP BY); htup_margin is
        gpusort_htup_margin.  projection_hash: list of Expr whose HashValue
        every projected row carries, written as kern_hashitems into a
        KDS_FORMAT_HASH kds_dst of proj_nslots slots (a pinned inner
        buffer)."""
        nrels = self.nrels
        blobs = {}
        self.htup_margin = htup_margin
        self.sort_limit = sort_limit
        self.join_inner_handle = join_inner_handle
        if sort_keys:
            blobs["gpusort"] = build_sort_keys(sort_keys, sort_window)
        if scan_quals is not None:
            blobs["scan"] = self.build_expr(scan_quals, 0)
        jq, hv = {}, {}
        for d, (hkeys, quals, others) in enumerate(joins, start=1):
            jq[d] = self.build_join_quals(quals, others, d)
            hv[d] = self.build_hash_value(hkeys, d)
        gdepth = nrels + 1
        # group-by key hash: SaveExpr(key) per key
        keyslots = []
        if groupby_keys:
            buf = _Buf()
            buf.b += bytearray(maxalign(40))
            for k in groupby_keys:
                keyslots.append(self.emit_save(buf, k, gdepth))
            head = _kexp_head(TOP("int4"), FOP("HashValue"), len(groupby_keys), 40)
            buf.b[:len(head)] = head
            buf.finish_kexp(0)
            blobs["keyhash"] = bytes(buf.b)
            # key load from kds_final (depth -2)
            nattrs = len(aggs) + len(groupby_keys)
            fin = []
            for i, k in enumerate(groupby_keys):
                d = KvDef(len(self.kvdefs), -2, len(aggs) + i + 1, k.typ, -1, -1, -1, ("final", i))
                self.kvdefs.append(d)
                fin.append(d)
            items = [(d.resno, d.slot) for d in fin]
            args_off = maxalign(48 + 4 * len(items))
            body = _kexp_head(TOP("int4"), FOP("LoadVars"), 0, args_off) + struct.pack("<ii", -2, len(items))
            body += b"".join(struct.pack("<hh", r, s) for r, s in items)
            b2 = _Buf()
            b2.b += body + b"\0" * (args_off - len(body))
            b2.finish_kexp(0)
            blobs["keyload"] = bytes(b2.b)
            # key compare
            cmp = _Buf()
            eqop = {"int2": "int2eq", "int4": "int4eq", "int8": "int8eq", "text": "text_eq",
                    "date": "date_eq", "float8": "float8eq", "numeric": "numeric_eq"}
            parts = []
            for ks, kf, k in zip(keyslots, fin, groupby_keys):
                b = _Buf()
                b.b += _kexp_head(TOP("bool"), FOP(eqop[k.typ]), 2, 40)
                p1 = b.append_aligned(_kexp_head(TOP(k.typ), FOP("VarExpr")) + struct.pack("<iH", -1, ks.slot))
                b.finish_kexp(p1)
                p2 = b.append_aligned(_kexp_head(TOP(k.typ), FOP("VarExpr")) + struct.pack("<iH", -1, kf.slot))
                b.finish_kexp(p2)
                b.finish_kexp(0)
                parts.append(bytes(b.b))
            if len(parts) == 1:
                blobs["keycomp"] = parts[0]
            else:
                b = _Buf()
                b.b += _kexp_head(TOP("bool"), FOP("BoolExpr_And"), len(parts), 40)
                for p in parts:
                    b.append_aligned(p)
                b.finish_kexp(0)
                blobs["keycomp"] = bytes(b.b)
        # AggFuncs
        nattrs = len(aggs) + len(groupby_keys)
        if nattrs:
            head_sz = maxalign(44 + 12 * nattrs)
            buf = _Buf()
            buf.b += bytearray(head_sz)
            descs = []
            nargs = 0
            used = set()
            for a in aggs:
                slots = []
                for arg in (a.arg, a.arg1):
                    slot = -1
                    if arg is not None:
                        pos = len(buf.b)
                        d = self.emit_save(buf, arg, gdepth)
                        slot = d.slot
                        if slot in used:
                            del buf.b[pos:]
                        else:
                            used.add(slot)
                            nargs += 1
                    slots.append(slot)
                descs.append((KAGG[a.action], slots[0], slots[1], -1, a.typmod))
            for k, ks in zip(groupby_keys, keyslots):
                pos = len(buf.b)
                d = self.emit_save(buf, k, gdepth)
                if d.slot in used:
                    del buf.b[pos:]
                else:
                    used.add(d.slot)
                    nargs += 1
                descs.append((KAGG["VREF"], d.slot, -1, -1, getattr(k, "typmod", -1)))
            head = _kexp_head(TOP("int4"), FOP("AggFuncs"), nargs, head_sz) + struct.pack("<i", nattrs)
            head += b"".join(struct.pack("<Hhhhi", *x) for x in descs)
            buf.b[:len(head)] = head
            buf.finish_kexp(0)
            blobs["actions"] = bytes(buf.b)
        if projection:
            blobs["projection"] = self.build_projection(projection, gdepth, projection_hash)
            dt = Table("kds_dst", [Column(f"c{i}", e.typ, getattr(e, "typmod", -1))
                                   for i, e in enumerate(projection)], 0)
            kd = dt.kds_header("h" if projection_hash else "r", 0)
            if projection_hash:
                struct.pack_into("<I", kd, 40, proj_nslots)     # hash_nslots
            blobs["kds_dst"] = bytes(kd)
        # LoadVars / MoveVars packed
        lv = {d: self.build_loadvars(d) for d in range(0, nrels + 1)}
        lv = {d: b for d, b in lv.items() if b is not None}
        blobs["loadvars"] = self.packed(lv, nrels + 1, nrels + 2) if lv else None
        mv = {d: self.build_movevars(d) for d in range(0, nrels + 1)}
        mv = {d: b for d, b in mv.items() if b is not None}
        blobs["movevars"] = self.packed(mv, nrels + 1, nrels + 1) if mv else None
        if joins:
            blobs["joinquals"] = self.packed(jq, nrels + 1, nrels + 1)
            blobs["hashvalues"] = self.packed(hv, nrels + 1, nrels + 1)
        # kds_final header for the partial-aggregation target list
        if nattrs:
            final_cols = []
            for a in aggs:
                if a.action in ("NROWS_ANY", "NROWS_COND"):
                    final_cols.append(Column("nrows", "int8"))
                else:
                    final_cols.append(Column("pagg", "bytea"))
            for i, k in enumerate(groupby_keys):
                final_cols.append(Column(f"key{i}", k.typ, getattr(k, "typmod", -1)))
            ft = Table("kds_final", final_cols, 0)
            if groupby_keys:
                kf = ft.kds_header("h", 0)
                struct.pack_into("<Q", kf, 0, 1 << 30)
            else:
                # an aggregate without GROUP BY keys: one tuple in a 4 MB
                # KDS_FORMAT_ROW buffer, no hash slots (executor.c:690-695)
                kf = ft.kds_header("r", 0)
                struct.pack_into("<Q", kf, 0, 4 << 20)
            blobs["kds_final"] = bytes(kf)
        return self._assemble(blobs, ngroups_estimate)

    def _assemble(self, blobs, ngroups_estimate):
        nparams = len(self.params)
        head_sz = maxalign(192 + 4 * max(nparams, 1))
        out = _Buf()
        out.b += bytearray(head_sz)
        offs = {}
        # kvars slot descriptors
        desc = b""
        for d in self.kvdefs:
            t = PGTYPES[d.typ]
            desc += struct.pack("<i?bhiiHHxxxxQ", TOP(d.typ), t.byval, t.attalign, t.attlen, d.typmod,
                                d.offset, 0, 0, 0)
        offs["kvars"] = out.append_aligned(desc) if desc else 0
        for key in ("loadvars", "movevars", "scan", "joinquals", "hashvalues",
                    "keyhash", "keyload", "keycomp", "actions", "kds_final",
                    "projection", "kds_dst", "gpusort"):
            b = blobs.get(key)
            offs[key] = out.append_aligned(b) if b else 0
        poffs = []
        for p in self.params:
            poffs.append(out.append_aligned(p) if p is not None else 0)
        b = out.b
        struct.pack_into("<QIIIIIIII", b, 0, 0x1234, len(self.kvdefs), len(self.kvdefs), offs["kvars"],
                         typealign(16, self.kvecs_usage), self.nrels + 1, 0, 0, self.flags)
        struct.pack_into("<q", b, 40, -1)
        struct.pack_into("<IIIIIIIIIIII", b, 48, offs["loadvars"], offs["movevars"], offs["scan"],
                         offs["joinquals"], offs["hashvalues"], 0, offs["projection"], offs["keyhash"],
                         offs["keyload"],
                         offs["keycomp"], offs["actions"], offs["gpusort"])
        struct.pack_into("<I", b, 128, offs["kds_dst"])
        struct.pack_into("<II", b, 152, getattr(self, "join_inner_handle", 0), offs["kds_final"])
        struct.pack_into("<Ii", b, 168, getattr(self, "htup_margin", 0), getattr(self, "sort_limit", 0))
        struct.pack_into("<If", b, 160, 0, float(ngroups_estimate))
        struct.pack_into("<I", b, 188, nparams)
        for i, p in enumerate(poffs):
            struct.pack_into("<I", b, 192 + 4 * i, p)
        return bytes(b)

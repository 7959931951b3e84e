"""
Decoder of a KDS_FORMAT_ROW buffer of projected rows (kds_dst) into Python
values, as PostgreSQL reads kern_tupitems back (KDS_GET_TUPITEM,
xpu_common.h:1337-1345, with the minimal-tuple layout of
__kern_form_minimal_tuple, xpu_common.cu:1096-1184).  Test and benchmark
infrastructure.
"""
import struct

import numpy as np

HEAP_HASNULL = 0x0001
OID_INT2, OID_INT4, OID_INT8, OID_FLOAT8 = 21, 23, 20, 701
OID_BOOL, OID_DATE, OID_TEXT, OID_BYTEA, OID_NUMERIC = 16, 1082, 25, 17, 1700


def kds_columns(b):
    """(attalign, attlen, atttypid) per column of a kern_data_store header."""
    ncols, = struct.unpack_from("<I", b, 20)
    cols = []
    for j in range(ncols):
        _, al, attlen, _, _, oid = struct.unpack_from("<?bhhhI", b, 72 + 168 * j)
        cols.append((max(al, 1), attlen, oid))
    return cols


def _varlena(b, p):
    """(payload, total bytes) of the varlena at p, 1- or 4-byte header."""
    if b[p] & 1:
        n = (b[p] >> 1) & 0x7F
        return b[p + 1:p + n], n
    n = struct.unpack_from("<I", b, p)[0] >> 2
    return b[p + 4:p + n], n


def decode_tuple(b, t, cols):
    """Values of the kern_tupitem at offset t (None for NULL); numeric is
    returned as its varlena bytes, text / bytea as their payload."""
    im2, im, t_hoff = struct.unpack_from("<HHB", b, t + 10)
    natts = im2 & 0x7FF
    hasnull = bool(im & HEAP_HASNULL)
    bits = b[t + 15:t + 15 + (natts + 7) // 8]
    pos = t_hoff - 8
    vals = []
    for j, (al, attlen, oid) in enumerate(cols):
        if j >= natts or (hasnull and not ((bits[j >> 3] >> (j & 7)) & 1)):
            vals.append(None)
            continue
        pos = (pos + al - 1) & ~(al - 1)
        p = t + pos
        if oid == OID_BOOL:
            vals.append(b[p] != 0); pos += 1
        elif oid == OID_INT2:
            vals.append(struct.unpack_from("<h", b, p)[0]); pos += 2
        elif oid in (OID_INT4, OID_DATE):
            vals.append(struct.unpack_from("<i", b, p)[0]); pos += 4
        elif oid == OID_FLOAT8:
            vals.append(struct.unpack_from("<d", b, p)[0]); pos += 8
        elif oid in (OID_TEXT, OID_BYTEA):
            payload, n = _varlena(b, p)
            vals.append(bytes(payload)); pos += n
        elif oid == OID_NUMERIC:
            _, n = _varlena(b, p)
            vals.append(bytes(b[p:p + n])); pos += n
        else:
            vals.append(struct.unpack_from("<q", b, p)[0]); pos += 8
    return vals


def decode_kds_rows(buf):
    """Returns (header, rows): header = dict(length, usage, nitems, format),
    rows = [(image without the trailing row id, row id, values)] in row
    index order."""
    b = bytes(buf) if not isinstance(buf, (bytes, bytearray)) else buf
    length, usage, nitems, ncols = struct.unpack_from("<QQII", b, 0)
    fmt = chr(b[24])
    nslots, = struct.unpack_from("<I", b, 40)
    nr_colmeta, = struct.unpack_from("<I", b, 68)
    head_len = (72 + 168 * nr_colmeta + 7) & ~7
    cols = kds_columns(b)
    rowidx = np.frombuffer(b, dtype=np.uint64, count=nitems, offset=head_len + 8 * nslots)
    rows = []
    for i in range(nitems):
        t = length - int(rowidx[i])
        t_len, = struct.unpack_from("<I", b, t)
        rowid, = struct.unpack_from("<I", b, t + t_len - 4)
        rows.append((bytes(b[t:t + t_len - 4]), rowid, decode_tuple(b, t, cols)))
    return {"length": length, "usage": usage, "nitems": nitems, "format": fmt}, rows

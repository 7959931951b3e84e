"""
Decoder of a kds_final buffer (KDS_FORMAT_HASH of partial-aggregation
tuples) into Python values, mirroring how PostgreSQL reads the tuples
(executor.c:861-883) and how aggfuncs.c interprets the kagg_state__*
records.  Test and benchmark infrastructure.
"""
import struct

import numpy as np

VREF, NROWS_ANY, NROWS_COND = 101, 201, 202
MINMAX_INT = (302, 303, 402, 403)
MINMAX_FP = (304, 404)
PSUM_INT = (501, 601)
PSUM_INT128 = (502, 602, 504, 604)
PSUM_FP = (503, 603)


def session_aggs(session: bytes):
    """[(action, arg0_slot, typmod)] of the session's AggFuncs, plus key types."""
    off_actions, = struct.unpack_from("<I", session, 88)
    if off_actions == 0:
        return []
    nattrs, = struct.unpack_from("<i", session, off_actions + 40)
    out = []
    for j in range(nattrs):
        action, a0, a1, flt, typmod = struct.unpack_from("<Hhhhi", session, off_actions + 44 + 12 * j)
        out.append((action, a0, typmod))
    return out


def slot_types(session: bytes):
    nslots, defs = struct.unpack_from("<II", session, 12)
    return [struct.unpack_from("<i", session, defs + 32 * i)[0] for i in range(nslots)]


def _i128(lo, hi):
    v = (hi << 64) | lo
    if v >= 1 << 127:
        v -= 1 << 128
    return v


def decode_kds_final(buf, session: bytes):
    """Returns {key_tuple: [state, ...]} with the aggregate states in
    target-list order (keys excluded)."""
    b = bytes(buf) if not isinstance(buf, (bytes, bytearray)) else bytes(buf)
    aggs = session_aggs(session)
    stypes = slot_types(session)
    length, usage, nitems, ncols = struct.unpack_from("<QQII", b, 0)
    nr_colmeta, = struct.unpack_from("<I", b, 68)
    nslots, = struct.unpack_from("<I", b, 40)
    head_len = (72 + 168 * nr_colmeta + 7) & ~7
    colalign = [struct.unpack_from("<b", b, 72 + 168 * j + 1)[0] for j in range(ncols)]
    rowidx = np.frombuffer(b, dtype=np.uint64, count=nitems, offset=head_len + 8 * nslots)
    out = {}
    for i in range(nitems):
        t = length - int(rowidx[i])
        t_len, h = struct.unpack_from("<II", b, t)
        im2, im, t_hoff = struct.unpack_from("<HHB", b, t + 10)
        natts = im2 & 0x7FF
        bits = b[t + 15:t + 15 + (natts + 7) // 8]
        pos = t_hoff - 8
        keys, states = [], []
        for j, (action, a0, typmod) in enumerate(aggs):
            isnull = not ((bits[j >> 3] >> (j & 7)) & 1)
            al = colalign[j]
            pos = (pos + al - 1) & ~(al - 1)
            p = t + pos
            if action == VREF:
                if isnull:
                    keys.append(None)
                    continue
                tc = stypes[a0]
                if tc in (11, 10):                      # text / bytea: 4B header here
                    hdr, = struct.unpack_from("<I", b, p)
                    n = hdr >> 2
                    keys.append(b[p + 4:p + n])
                    pos += n
                elif tc == 9:                            # numeric varlena as-is
                    n = (b[p] >> 1) & 0x7F if b[p] & 1 else struct.unpack_from("<I", b, p)[0] >> 2
                    keys.append(b[p:p + n])
                    pos += n
                elif tc == 3:
                    keys.append(struct.unpack_from("<h", b, p)[0]); pos += 2
                elif tc in (4, 13):
                    keys.append(struct.unpack_from("<i", b, p)[0]); pos += 4
                elif tc == 1:
                    keys.append(b[p]); pos += 1
                elif tc == 8:
                    keys.append(struct.unpack_from("<d", b, p)[0]); pos += 8
                else:
                    keys.append(struct.unpack_from("<q", b, p)[0]); pos += 8
                continue
            if action in (NROWS_ANY, NROWS_COND):
                states.append(struct.unpack_from("<q", b, p)[0]); pos += 8
            elif action in MINMAX_INT:
                _, attrs, v = struct.unpack_from("<iIq", b, p)
                states.append((attrs & 1, v)); pos += 16
            elif action in MINMAX_FP:
                _, attrs, v = struct.unpack_from("<iId", b, p)
                states.append((attrs & 1, v)); pos += 16
            elif action in PSUM_INT:
                _, attrs, n, s = struct.unpack_from("<iIqq", b, p)
                states.append((n, s)); pos += 24
            elif action in PSUM_FP:
                _, attrs, n, s = struct.unpack_from("<iIqd", b, p)
                states.append((n, s)); pos += 24
            elif action in PSUM_INT128:
                _, attrs, n, lo, hi = struct.unpack_from("<iIQQQ", b, p)
                if action in (504, 604):
                    states.append((n, _i128(lo, hi), attrs & 0xFFFF))
                else:
                    states.append((n, _i128(lo, hi)))
                pos += 32
            elif action == 701:
                _, attrs, n, sx, sx2 = struct.unpack_from("<iIqdd", b, p)
                states.append((n, sx, sx2)); pos += 32
            elif action == 801:
                vals = struct.unpack_from("<iIqddddd", b, p)
                states.append(tuple(vals[2:])); pos += 56
            else:
                raise ValueError(f"unknown action {action}")
        out[tuple(keys)] = states
    return out


class Approx(float):
    """An expected float sum with the sum of its terms' magnitudes: a sum
    whose terms cancel is only defined to rtol of that magnitude (the
    row-ordered FP64 sum itself carries n * eps * sum|x| of error)."""

    def __new__(cls, value, scale):
        obj = super().__new__(cls, value)
        obj.scale = float(scale)
        return obj


def compare_groups(got, want, rtol=1e-12):
    """Integer / numeric states exact, float states within rtol relative
    (relative to the sum of magnitudes when the expected value is an
    Approx).  Returns a list of mismatch descriptions (empty when equal)."""
    errs = []
    if set(got) != set(want):
        errs.append(f"group keys differ: only-got={sorted(set(got) - set(want))[:5]} "
                    f"only-want={sorted(set(want) - set(got))[:5]}")
        return errs
    for k in want:
        g, w = got[k], want[k]
        if len(g) != len(w):
            errs.append(f"{k}: {len(g)} states vs {len(w)}")
            continue
        for j, (x, y) in enumerate(zip(g, w)):
            if isinstance(y, tuple):
                for xe, ye in zip(x, y):
                    if ye is None:              # undefined (e.g. min of no rows)
                        continue
                    if isinstance(ye, float):
                        tol = rtol * max(abs(ye), getattr(ye, "scale", 0.0), 1e-300)
                        if not (abs(xe - ye) <= tol or xe == ye):
                            errs.append(f"{k}[{j}]: float {xe!r} vs {ye!r}")
                    elif xe != ye:
                        errs.append(f"{k}[{j}]: {xe!r} vs {ye!r}")
            elif x != y:
                errs.append(f"{k}[{j}]: {x!r} vs {y!r}")
    return errs


# ---------------------------------------------------------------------------
# GPU-Sort restated: the order of final groups by SortKeys (the comparators
# and prep functions of cuda_gpusort.cu:15-400), LIMIT and window ranks
# (cuda_gpusort.cu:816-996), over decoded groups
# ---------------------------------------------------------------------------
def sort_key_values(row, session, sort_keys):
    """The SQL value (None for NULL) of each sort key of one decoded group
    (key tuple, states); sort_keys as given to build_sort_keys."""
    import math
    keys, states = row
    aggs = session_aggs(session)
    out = []
    for kind, anum, _asc, _nf in sort_keys:
        action = aggs[anum - 1][0]
        if action == VREF:
            out.append(keys[sum(1 for a in aggs[:anum - 1] if a[0] == VREF)])
            continue
        st = states[sum(1 for a in aggs[:anum - 1] if a[0] != VREF)]
        if kind == "VREF":
            out.append(st)
        elif kind in ("PMINMAX_INT64", "PMINMAX_FP64"):
            out.append(st[1] if st[0] else None)
        elif kind in ("PSUM_INT64", "PSUM_NUMERIC", "PSUM_FP64"):
            out.append(st[1] if st[0] else None)
        elif kind in ("PAVG_INT64", "PAVG_FP64", "PAVG_NUMERIC"):
            out.append(float(st[1]) / st[0] if st[0] else None)
        elif kind in ("PVARIANCE_SAMP", "PVARIANCE_POP"):
            n, sx, sxx = st
            samp = kind == "PVARIANCE_SAMP"
            if n < (2 if samp else 1):
                out.append(None)
            else:
                num = max(n * sxx - sx * sx, 0.0)
                out.append(num / (n * (n - 1 if samp else n)))
        elif kind.startswith("PCOVAR_"):
            n, sx, sxx, sy, syy, sxy = st
            if kind == "PCOVAR_COUNT":
                out.append(float(n))
            elif n < 1 or (kind == "PCOVAR_SAMP" and n < 2):
                out.append(None)
            elif kind == "PCOVAR_AVGX":
                out.append(sx / n)
            elif kind == "PCOVAR_AVGY":
                out.append(sy / n)
            elif kind == "PCOVAR_POP":
                out.append((sxy - sx * sy / n) / n)
            elif kind == "PCOVAR_SAMP":
                out.append((sxy - sx * sy / n) / (n - 1))
            else:
                vx, vy = n * sxx - sx * sx, n * syy - sy * sy
                out.append(None if vx <= 0 or vy <= 0 else (n * sxy - sx * sy) / math.sqrt(vx * vy))
        elif kind == "NITEMS":
            out.append(st[0])
        else:
            raise ValueError(kind)
    return out


def _cmp_values(a, b, sort_keys):
    for (kind, _anum, asc, nulls_first), x, y in zip(sort_keys, a, b):
        if x is None or y is None:
            if x is None and y is None:
                continue
            xn = x is None
            return (-1 if xn else 1) if nulls_first else (1 if xn else -1)
        if x != y:
            c = -1 if x < y else 1
            return c if asc else -c
    return 0


def order_groups(rows, session, sort_keys, window=None, limit=0):
    """Expected output of a GPU-Sort Final: the decoded groups (key tuple,
    states) in sort order, cut by LIMIT or filtered by the window rank
    (window = (function 'n' / 'r' / 'd', partition keys, order keys,
    rank limit)).  Rows with equal sort keys may come in any order."""
    import functools
    vals = [(sort_key_values(r, session, sort_keys), r) for r in rows]
    vals.sort(key=functools.cmp_to_key(lambda a, b: _cmp_values(a[0], b[0], sort_keys)))
    if window:
        wf, pb, ob, lim = window
        out, ps, peer, dense = [], 0, 0, 0
        for p, (v, r) in enumerate(vals):
            if p == 0 or _cmp_values(v[:pb], vals[p - 1][0][:pb], sort_keys[:pb]) != 0:
                ps, peer, dense = p, p, 1
            elif _cmp_values(v[pb:pb + ob], vals[p - 1][0][pb:pb + ob], sort_keys[pb:pb + ob]) != 0:
                peer, dense = p, dense + 1
            rank = {"n": p - ps + 1, "r": peer - ps + 1, "d": dense}[wf]
            if lim == 0 or rank <= lim:
                out.append((v, r))
        vals = out
    elif limit > 0:
        vals = vals[:limit]
    return vals

"""
Seeded synthetic workloads with the shapes, sizes and value distributions of
the benchmark configurations (test and benchmark infrastructure).

  scan_groupby     heap table (id int8, a int4 U[0,1000), b float8 N(0,1)
                   with 5% NULL, c numeric(12,2) U[0,10000), g int4 U[0,64));
                   WHERE a < 300 GROUP BY g -> count(*), sum(a), sum(c), avg(b)
  join_groupby     fact(fk1, fk2, qty int4 U[1,50], price int8 U[100,1e6])
                   with fk1 U[1,200000] into dim1(pk int4, region text: 25
                   values of 8-16 bytes) and fk2 bounded-Zipf(s=1.1) over
                   1..10000 into dim2(pk int4, flag int2 in 0..4);
                   JOIN dim1, dim2 WHERE flag < 3 GROUP BY region ->
                   sum(qty*price), count(*)
  mixed_commands   batched chunk commands on the scan_groupby schema: chunk
                   sizes log-uniform, selectivity (a < t) uniform, group
                   counts (the domain of g) log-uniform, one session each
  scan_projection  the scan_groupby table, WHERE a < 300 projected to
                   (id, a, b, c, a * 2 + g) rows (no GROUP BY)
  join_projection  the join_groupby tables, projected to
                   (fk1, qty * price, region, flag) rows

Every generator also returns the expected per-group aggregates computed
directly from the column arrays with numpy (independent of any page or
bytecode decoding), so the oracle itself can be pinned against them.
"""
import struct

import numpy as np

from xb_final import Approx
from xb_producer import (BLCKSZ, Table, Column, Var, Const, Func, Agg, SessionBuilder,
                         encode_numeric, encode_varlena_list, encode_numeric_array, encode_text_array, encode_text_from_dict,
                         hash_u32_array, hash_merge_array, kern_multirels, numeric_typmod)

DEVKIND_GPU = 0x00000001
DEVTASK_SCAN = 0x10000000
DEVTASK_JOIN = 0x20000000
DEVTASK_PREAGG = 0x40000000

SEED_BASE = 0x5EED0000


def rng_for(config, table):
    return np.random.Generator(np.random.PCG64(SEED_BASE + config * 16 + table))


def host_join_hash_int4(keys: np.ndarray) -> np.ndarray:
    """get_tuple_hashvalue for one int4 key (gpu_join.c:1549-1584)."""
    h = hash_merge_array(np.full(len(keys), 0xFFFFFFFF, dtype=np.uint32), hash_u32_array(keys, 4))
    return h ^ np.uint32(0xFFFFFFFF)


# ---------------------------------------------------------------------------
def scan_groupby_session(a_limit=300, ngroups=64):
    """WHERE a < a_limit GROUP BY g -> count(*), sum(a), sum(c), avg(b)."""
    typmod_c = numeric_typmod(12, 2)
    va, vb, vc, vg = (Var(0, 2, "int4"), Var(0, 3, "float8"),
                      Var(0, 4, "numeric", typmod_c), Var(0, 5, "int4"))
    sb = SessionBuilder(0, DEVTASK_PREAGG | DEVKIND_GPU)
    return sb.build(
        scan_quals=Func("int4lt", [va, Const("int4", a_limit)], "bool"),
        groupby_keys=[vg],
        aggs=[Agg("NROWS_ANY"),
              Agg("PSUM_INT", Func("int4_to_int8", [va], "int8")),
              Agg("PSUM_NUMERIC", vc, typmod_c),
              Agg("PAVG_FP", vb)],
        ngroups_estimate=float(ngroups))


def _scan_table(nrows, seed_config, null_frac, ngroups):
    """t0 (id int8, a int4, b float8 with NULLs, c numeric(12,2), g int4)
    and its column arrays."""
    r = rng_for(seed_config, 0)
    id_ = np.arange(nrows, dtype=np.int64)
    a = r.integers(0, 1000, nrows, dtype=np.int32)
    b = r.standard_normal(nrows)
    bnull = r.random(nrows) < null_frac
    c_unscaled = r.integers(0, 1_000_000, nrows, dtype=np.int64)
    g = r.integers(0, ngroups, nrows, dtype=np.int32)
    typmod_c = numeric_typmod(12, 2)
    tbl = Table("t0", [
        Column("id", "int8", values=id_),
        Column("a", "int4", values=a),
        Column("b", "float8", values=b, nulls=bnull),
        Column("c", "numeric", typmod=typmod_c, values=encode_numeric_array(c_unscaled, 2)),
        Column("g", "int4", values=g),
    ], nrows)
    return tbl, a, b, bnull, c_unscaled, g


def scan_groupby(nrows=4_000_000, seed_config=0, null_frac=0.05, a_limit=300, ngroups=64):
    """The plain scan + filter + group-by table; ngroups sets the domain of
    g (64 in the benchmark configuration)."""
    tbl, a, b, bnull, c_unscaled, g = _scan_table(nrows, seed_config, null_frac, ngroups)
    session = scan_groupby_session(a_limit, ngroups)
    expect, meta = _scan_expect(a, b, bnull, c_unscaled, g, a_limit, ngroups)
    return tbl, session, None, expect, meta


def _scan_expect(a, b, bnull, c_unscaled, g, a_limit, ngroups, visible=None):
    """expected partial states per group of scan_groupby_session, straight
    from the arrays; visible masks the rows the chunks still hold"""
    nrows = len(a)
    m = a < a_limit
    if visible is not None:
        m &= visible
    gm = g[m]
    cnt = np.bincount(gm, minlength=ngroups)
    sa = np.zeros(ngroups, dtype=np.int64)
    np.add.at(sa, gm, a[m].astype(np.int64))
    sc = np.zeros(ngroups, dtype=np.int64)
    np.add.at(sc, gm, c_unscaled[m])
    mb = m & ~bnull
    sb_ = np.zeros(ngroups, dtype=np.float64)
    np.add.at(sb_, g[mb], b[mb])                 # unbuffered: row order per group
    nb = np.bincount(g[mb], minlength=ngroups)
    sab = np.zeros(ngroups, dtype=np.float64)
    np.add.at(sab, g[mb], np.abs(b[mb]))
    expect = {}
    for k in np.flatnonzero(cnt).tolist():
        expect[(k,)] = {"nrows": int(cnt[k]), "sum_a": (int(cnt[k]), int(sa[k])),
                        "sum_c": (int(cnt[k]), int(sc[k]), 2),
                        "avg_b": (int(nb[k]), Approx(float(sb_[k]), float(sab[k])))}
    meta = {"nitems_raw": nrows if visible is None else int(visible.sum()),
            "nitems_in": int(m.sum()), "nitems_out": int(m.sum()),
            "agg_names": ["nrows", "sum_a", "sum_c", "avg_b"], "nkeys": 1}
    return expect, meta


LP_UNUSED, LP_NORMAL, LP_REDIRECT, LP_DEAD = 0, 1, 2, 3


def invalidate_lines(chunks, frac, seed=41):
    """Copies of KDS_FORMAT_BLOCK chunks in which a share 'frac' of the line
    pointers no longer point at a visible tuple, the pages the reference's
    relscan.c hands the GPU when they are not all-visible (it sets the line
    pointers of invisible tuples unused, src/relscan.c:462-494), and pages
    after HOT pruning (dead items keeping their storage, redirects).  Each
    chosen line pointer becomes LP_UNUSED (offset and length cleared),
    LP_DEAD (storage kept) or LP_REDIRECT (offset = another line number,
    length 0), in turn.  Returns the chunks and the mask of rows, in the
    order the chunks hold them, that stay visible."""
    r = np.random.default_rng(seed)
    out, keep = [], []
    kind = 0
    for ch in chunks:
        ch = ch.copy()
        nblocks, = struct.unpack_from("<I", ch, 16)
        block_offset, = struct.unpack_from("<I", ch, 44)
        for b in range(nblocks):
            base = block_offset + b * BLCKSZ
            lower, = struct.unpack_from("<H", ch, base + 12)
            nlp = (lower - 24) // 4
            for i in range(nlp):
                pos = base + 24 + 4 * i
                lp, = struct.unpack_from("<I", ch, pos)
                if ((lp >> 15) & 3) != LP_NORMAL:
                    continue
                if r.random() >= frac:
                    keep.append(True)
                    continue
                keep.append(False)
                if kind == 0:
                    lp = 0
                elif kind == 1:
                    lp = (lp & ~(3 << 15)) | (LP_DEAD << 15)
                else:
                    lp = (((i + 1) % nlp) + 1) | (LP_REDIRECT << 15)
                kind = (kind + 1) % 3
                struct.pack_into("<I", ch, pos, lp)
        out.append(ch)
    return out, np.array(keep, dtype=bool)


def scan_groupby_filtered(nrows=200_000, seed_config=40, null_frac=0.05, a_limit=300, ngroups=64,
                          pages_per_chunk=200, frac=0.15):
    """scan_groupby over pages whose line pointers are partly invalidated
    (invalidate_lines).  Returns (chunks, session, expect, meta) with the
    expected groups over the rows left visible."""
    tbl, a, b, bnull, c_unscaled, g = _scan_table(nrows, seed_config, null_frac, ngroups)
    session = scan_groupby_session(a_limit, ngroups)
    chunks, keep = invalidate_lines(tbl.block_chunks(pages_per_chunk=pages_per_chunk), frac,
                                    seed=seed_config + 1)
    assert len(keep) == nrows
    expect, meta = _scan_expect(a, b, bnull, c_unscaled, g, a_limit, ngroups, visible=keep)
    return chunks, session, expect, meta


def wide_groupby_session(a_limit=600, ngroups=3000, sort=None):
    """WHERE a < a_limit GROUP BY g -> count(*), count(b), min(a),
    max(a::int8), min(b), max(b), sum(b), avg(c), stddev(b), covar(b, a):
    every partial state form of kds_final (attributes 1..10, g is 11).
    sort: dict(keys=[(kind, attribute, asc, nulls_first)], window=(func,
    partition keys, order keys, rank limit), limit=n) for a GPU-Sort of the
    groups at Final."""
    typmod_c = numeric_typmod(12, 2)
    va, vb, vc, vg = (Var(0, 2, "int4"), Var(0, 3, "float8"),
                      Var(0, 4, "numeric", typmod_c), Var(0, 5, "int4"))
    sb = SessionBuilder(0, DEVTASK_PREAGG | DEVKIND_GPU)
    return sb.build(
        scan_quals=Func("int4lt", [va, Const("int4", a_limit)], "bool"),
        groupby_keys=[vg],
        aggs=[Agg("NROWS_ANY"),
              Agg("NROWS_COND", vb),
              Agg("PMIN_INT32", va),
              Agg("PMAX_INT64", Func("int4_to_int8", [va], "int8")),
              Agg("PMIN_FP64", vb),
              Agg("PMAX_FP64", vb),
              Agg("PSUM_FP", vb),
              Agg("PAVG_NUMERIC", vc, typmod_c),
              Agg("STDDEV", vb),
              Agg("COVAR", vb, arg1=Func("int4_to_float8", [va], "float8"))],
        ngroups_estimate=float(ngroups),
        **_sort_args(sort))


def scan_nogroup_session(a_limit=300):
    """WHERE a < a_limit -> count(*), count(b), sum(a), sum(c), avg(b),
    min(b), max(b): an aggregate without GROUP BY keys (one result tuple,
    KDS_FORMAT_ROW kds_final).  max(float8) is the state the reference's
    no-group global-memory path updates with an atomic minimum
    (cuda_gpupreagg.cu:524-526); the SQL result is the maximum."""
    typmod_c = numeric_typmod(12, 2)
    va, vb, vc = Var(0, 2, "int4"), Var(0, 3, "float8"), Var(0, 4, "numeric", typmod_c)
    sb = SessionBuilder(0, DEVTASK_PREAGG | DEVKIND_GPU)
    return sb.build(
        scan_quals=Func("int4lt", [va, Const("int4", a_limit)], "bool"),
        groupby_keys=[],
        aggs=[Agg("NROWS_ANY"),
              Agg("NROWS_COND", vb),
              Agg("PSUM_INT", Func("int4_to_int8", [va], "int8")),
              Agg("PSUM_NUMERIC", vc, typmod_c),
              Agg("PAVG_FP", vb),
              Agg("PMIN_FP64", vb),
              Agg("PMAX_FP64", vb)],
        ngroups_estimate=1.0)


def scan_nogroup(nrows=4_000_000, seed_config=0, null_frac=0.05, a_limit=300):
    """The plain scan table under scan_nogroup_session, with the one
    expected result tuple (key ()) computed from the column arrays; no
    tuple at all when no row qualifies."""
    tbl, a, b, bnull, c_unscaled, g = _scan_table(nrows, seed_config, null_frac, 64)
    session = scan_nogroup_session(a_limit)
    m = a < a_limit
    mb = m & ~bnull
    n, nb = int(m.sum()), int(mb.sum())
    expect = {}
    if n:
        bs = b[mb]
        fsum = 0.0
        for x in bs:                                # row-ordered FP64 sum
            fsum += float(x)
        valid = 1 if nb else 0
        expect[()] = [n, nb, (n, int(a[m].astype(np.int64).sum())), (n, int(c_unscaled[m].sum()), 2),
                      (nb, Approx(fsum, float(np.abs(bs).sum()))),
                      (valid, float(bs.min()) if nb else None), (valid, float(bs.max()) if nb else None)]
    meta = {"nitems_raw": nrows, "nitems_in": n, "nitems_out": n, "nkeys": 0}
    return tbl, session, None, expect, meta


def long_strings(n, seed=7, lo=20, hi=300):
    """n distinct strings whose lengths straddle the 1-byte varlena limit:
    the first ones are 1, 126, 127, 128 and 300 bytes long (126 is the
    longest payload of a 1-byte header), the rest uniform in [lo, hi]."""
    r = np.random.Generator(np.random.PCG64(seed))
    fixed = [1, 126, 127, 128, 300]
    lens = fixed[:n] + r.integers(lo, hi + 1, max(0, n - len(fixed))).tolist()
    # letters stepping by 3 through the alphabet, from a per-string offset
    pat = "".join(chr(97 + (3 * k) % 26) for k in range(26)) * (hi // 26 + 14)
    out = []
    for i, L in enumerate(lens):
        head = "%d:" % i
        off = (63 * i) % 26
        body = pat[off:off + L]
        out.append((head + body)[:L] if L > len(head) else chr(65 + i % 26) * L)
    assert len(set(out)) == n
    return out


def long_varlena_session(v_limit=700, ngroups=150):
    """WHERE v < v_limit GROUP BY t -> count(*), count(n), sum(n), avg(n),
    sum(v) over (id int8, t text, n numeric(18,4), v int4)."""
    typmod_n = numeric_typmod(18, 4)
    vt, vn, vv = Var(0, 2, "text"), Var(0, 3, "numeric", typmod_n), Var(0, 4, "int4")
    sb = SessionBuilder(0, DEVTASK_PREAGG | DEVKIND_GPU)
    return sb.build(
        scan_quals=Func("int4lt", [vv, Const("int4", v_limit)], "bool"),
        groupby_keys=[vt],
        aggs=[Agg("NROWS_ANY"), Agg("NROWS_COND", vn),
              Agg("PSUM_NUMERIC", vn, typmod_n), Agg("PAVG_NUMERIC", vn, typmod_n),
              Agg("PSUM_INT", Func("int4_to_int8", [vv], "int8"))],
        ngroups_estimate=float(ngroups))


def long_varlena_groupby(nrows=100_000, ngroups=150, seed_config=6, null_frac=0.03, v_limit=700):
    """Heap table (id int8, t text, n numeric(18,4), v int4) whose varlenas
    take every on-disk form the heap decoder must read: t is one of
    ngroups strings of 1..300 bytes (those above 126 bytes carry a 4-byte
    header, aligned to 4 in the tuple); n is U(-1e8, 1e8) at 4 decimals
    with 3% NULLs, one third in the short numeric format, one third in the
    NUMERIC_LONG format (n_sign_dscale + n_weight), one third in the long
    format with a 4-byte varlena header.  Expected states from the
    arrays."""
    r = rng_for(seed_config, 0)
    words = long_strings(ngroups, seed=SEED_BASE + seed_config)
    code = r.integers(0, ngroups, nrows)
    v = r.integers(0, 1000, nrows, dtype=np.int32)
    n_unscaled = r.integers(-10 ** 12, 10 ** 12, nrows, dtype=np.int64)
    nnull = r.random(nrows) < null_frac
    form = r.integers(0, 3, nrows)
    nimg = [encode_numeric(int(x), 4, long_fmt=f >= 1, hdr4=f == 2)
            for x, f in zip(n_unscaled.tolist(), form.tolist())]
    typmod_n = numeric_typmod(18, 4)
    tbl = Table("t6", [
        Column("id", "int8", values=np.arange(nrows, dtype=np.int64)),
        Column("t", "text", values=encode_text_from_dict(code, words)),
        Column("n", "numeric", typmod=typmod_n, values=encode_varlena_list(nimg), nulls=nnull),
        Column("v", "int4", values=v),
    ], nrows)
    session = long_varlena_session(v_limit, ngroups)
    m = v < v_limit
    mn = m & ~nnull
    cnt = np.bincount(code[m], minlength=ngroups)
    cn = np.bincount(code[mn], minlength=ngroups)
    sv = np.zeros(ngroups, dtype=np.int64)
    np.add.at(sv, code[m], v[m].astype(np.int64))
    sn = [0] * ngroups
    for k, x in zip(code[mn].tolist(), n_unscaled[mn].tolist()):
        sn[k] += x
    expect = {}
    for k in np.flatnonzero(cnt).tolist():
        expect[(words[k].encode(),)] = [int(cnt[k]), int(cn[k]), (int(cn[k]), sn[k], 4), (int(cn[k]), sn[k], 4),
                                        (int(cnt[k]), int(sv[k]))]
    meta = {"nitems_raw": nrows, "nitems_in": int(m.sum()), "nitems_out": int(m.sum()), "nkeys": 1,
            "words": words}
    return tbl, session, None, expect, meta


def _sort_args(sort):
    if not sort:
        return {}
    return {"sort_keys": sort["keys"], "sort_window": sort.get("window"), "sort_limit": sort.get("limit", 0)}


def _group_sum(g, m, x, n):
    out = np.zeros(n, dtype=np.float64)
    np.add.at(out, g[m], x[m])                   # unbuffered: row order per group
    return out


def wide_groupby(nrows=200_000, seed_config=5, null_frac=0.05, a_limit=600, ngroups=3000):
    """The scan table under wide_groupby_session, with the expected
    partial states per group (float sums as Approx with their terms'
    magnitude)."""
    tbl, a, b, bnull, c_unscaled, g = _scan_table(nrows, seed_config, null_frac, ngroups)
    session = wide_groupby_session(a_limit, ngroups)
    m = a < a_limit
    mb = m & ~bnull
    cnt = np.bincount(g[m], minlength=ngroups)
    nb = np.bincount(g[mb], minlength=ngroups)
    amin = np.full(ngroups, np.iinfo(np.int64).max)
    np.minimum.at(amin, g[m], a[m].astype(np.int64))
    amax = np.full(ngroups, np.iinfo(np.int64).min)
    np.maximum.at(amax, g[m], a[m].astype(np.int64))
    bmin = np.full(ngroups, np.inf)
    np.minimum.at(bmin, g[mb], b[mb])
    bmax = np.full(ngroups, -np.inf)
    np.maximum.at(bmax, g[mb], b[mb])
    sc = np.zeros(ngroups, dtype=np.int64)
    np.add.at(sc, g[m], c_unscaled[m])
    af = a.astype(np.float64)
    sx, sax = _group_sum(g, mb, b, ngroups), _group_sum(g, mb, np.abs(b), ngroups)
    sxx = _group_sum(g, mb, b * b, ngroups)
    sy, syy = _group_sum(g, mb, af, ngroups), _group_sum(g, mb, af * af, ngroups)
    sxy, saxy = _group_sum(g, mb, b * af, ngroups), _group_sum(g, mb, np.abs(b * af), ngroups)
    expect = {}
    for k in np.flatnonzero(cnt).tolist():
        valid = 1 if nb[k] else 0
        expect[(k,)] = [
            int(cnt[k]), int(nb[k]),
            (1, int(amin[k])), (1, int(amax[k])),
            (valid, float(bmin[k]) if valid else None), (valid, float(bmax[k]) if valid else None),
            (int(nb[k]), Approx(float(sx[k]), float(sax[k]))),
            (int(cnt[k]), int(sc[k]), 2),
            (int(nb[k]), Approx(float(sx[k]), float(sax[k])), Approx(float(sxx[k]), float(sxx[k]))),
            (int(nb[k]), Approx(float(sx[k]), float(sax[k])), Approx(float(sxx[k]), float(sxx[k])),
             Approx(float(sy[k]), float(sy[k])), Approx(float(syy[k]), float(syy[k])),
             Approx(float(sxy[k]), float(saxy[k]))),
        ]
    meta = {"nitems_raw": nrows, "nitems_in": int(m.sum()), "nitems_out": int(m.sum()), "nkeys": 1}
    return tbl, session, None, expect, meta


REGIONS = [("region_%02d" % i) + "abcdefg"[: (i * 3) % 8] for i in range(25)]


def zipf_bounded(r, n, s, size):
    """Bounded Zipf over 1..n with exponent s via its explicit CDF."""
    w = 1.0 / np.arange(1, n + 1, dtype=np.float64) ** s
    cdf = np.cumsum(w)
    cdf /= cdf[-1]
    u = r.random(size)
    return (np.searchsorted(cdf, u, side="right") + 1).astype(np.int32)


def join_groupby_session(flag_limit=3, sort=None, inner_handle=0):
    """fact JOIN dim1 ON fk1 = pk JOIN dim2 ON fk2 = pk AND flag < flag_limit
    GROUP BY region -> sum(qty * price), count(*)."""
    f_fk1, f_fk2, f_qty, f_price = (Var(0, 1, "int4"), Var(0, 2, "int4"),
                                    Var(0, 3, "int4"), Var(0, 4, "int8"))
    d1_pk, d1_region = Var(1, 1, "int4"), Var(1, 2, "text")
    d2_pk, d2_flag = Var(2, 1, "int4"), Var(2, 2, "int2")
    sb = SessionBuilder(2, DEVTASK_JOIN | DEVTASK_PREAGG | DEVKIND_GPU)
    return sb.build(
        joins=[([f_fk1], [Func("int4eq", [f_fk1, d1_pk], "bool")], []),
               ([f_fk2], [Func("int4eq", [f_fk2, d2_pk], "bool")],
                [Func("int24lt", [d2_flag, Const("int4", flag_limit)], "bool")])],
        groupby_keys=[d1_region],
        aggs=[Agg("PSUM_INT64", Func("int48mul", [f_qty, f_price], "int8")),
              Agg("NROWS_ANY")],
        ngroups_estimate=25.0, join_inner_handle=inner_handle,
        **_sort_args(sort))


def join_groupby(nfact=100_000_000, ndim1=200_000, ndim2=10_000, seed_config=1, flag_limit=3,
                 key_stride=1, dim1_copies=1, miss_frac=0.0, with_rows=False, price_hi=1_000_000,
                 regions=None):
    """Two-way hash join + group-by.  Defaults give the headline workload:
    dense unique dimension keys 1..n, every fact row matching.  Variants for
    the join paths: key_stride spreads the keys (k * stride; sparse keys
    take the hashed probe instead of direct addressing), dim1_copies > 1
    repeats every dim1 key with its own region (several matches per probe),
    miss_frac makes that share of fact rows reference no dim1 row.
    with_rows adds meta["rows"]: the sorted (fk1, qty * price, region,
    flag) tuples of every joined row.regions replaces the 25 region strings (e.g. strings longer than 126
    bytes, whose varlena header is 4 bytes).
    """
    REG = REGIONS if regions is None else regions
    r1 = rng_for(seed_config, 1)
    r2 = rng_for(seed_config, 2)
    rf = rng_for(seed_config, 0)
    # dimensions
    pk1_one = np.arange(1, ndim1 + 1, dtype=np.int64) * key_stride
    pk1 = np.tile(pk1_one, dim1_copies).astype(np.int32)
    reg_code = r1.integers(0, len(REG), ndim1 * dim1_copies)
    dim1 = Table("dim1", [Column("pk", "int4", values=pk1),
                          Column("region", "text", values=encode_text_from_dict(reg_code, REG))],
                 ndim1 * dim1_copies)
    pk2 = (np.arange(1, ndim2 + 1, dtype=np.int64) * key_stride).astype(np.int32)
    flag = r2.integers(0, 5, ndim2, dtype=np.int16)
    dim2 = Table("dim2", [Column("pk", "int4", values=pk2), Column("flag", "int2", values=flag)], ndim2)
    # fact
    fk1 = rf.integers(1, ndim1 + 1, nfact, dtype=np.int32)
    fk2 = zipf_bounded(rf, ndim2, 1.1, nfact)
    qty = rf.integers(1, 51, nfact, dtype=np.int32)
    price = rf.integers(100, price_hi + 1, nfact, dtype=np.int64)
    idx1 = fk1.astype(np.int64) - 1
    idx2 = fk2.astype(np.int64) - 1
    miss = np.zeros(nfact, dtype=bool)
    if miss_frac > 0:
        miss = rf.random(nfact) < miss_frac
        fk1 = np.where(miss, fk1 + ndim1, fk1).astype(np.int32)     # beyond every dim1 key
    if key_stride != 1:
        fk1 = (fk1.astype(np.int64) * key_stride).astype(np.int32)
        fk2 = (fk2.astype(np.int64) * key_stride).astype(np.int32)
    fact = Table("fact", [Column("fk1", "int4", values=fk1), Column("fk2", "int4", values=fk2),
                          Column("qty", "int4", values=qty), Column("price", "int8", values=price)], nfact)
    kmrels = kern_multirels([dim1.hash_kds(host_join_hash_int4(pk1)),
                             dim2.hash_kds(host_join_hash_int4(pk2))])
    dims = {"dim1": dim1, "dim2": dim2, "pk1": pk1, "pk2": pk2}
    session = join_groupby_session(flag_limit)
    # expected: every (fact row, dim1 copy) pair that passes both joins
    m = (flag[idx2] < flag_limit) & ~miss
    amount = qty.astype(np.int64) * price
    cnt = np.zeros(len(REG), dtype=np.int64)
    tot = [0] * len(REG)
    for c in range(dim1_copies):
        region_row = reg_code[c * ndim1 + idx1]
        for k in range(len(REG)):
            sel = m & (region_row == k)
            cnt[k] += int(sel.sum())
            tot[k] += int(amount[sel].sum())
    expect = {}
    for k in range(len(REG)):
        if cnt[k]:
            expect[(REG[k].encode(),)] = {"sum_amount": (int(cnt[k]), tot[k]), "nrows": int(cnt[k])}
    if with_rows:
        rows = []
        sel = np.flatnonzero(m)
        for c in range(dim1_copies):
            region_row = reg_code[c * ndim1 + idx1[sel]]
            rows += list(zip(fk1[sel].tolist(), amount[sel].tolist(),
                             [REG[k].encode() for k in region_row], flag[idx2[sel]].tolist()))
        rows.sort()
    hit1 = int((~miss).sum()) * dim1_copies
    out = int(m.sum()) * dim1_copies
    meta = {"nitems_raw": nfact, "nitems_in": nfact, "nitems_out": out,
            "depth_out": [hit1, out], "agg_names": ["sum_amount", "nrows"], "nkeys": 1}
    if with_rows:
        meta["rows"] = rows
    meta["dims"] = dims
    return fact, session, kmrels, expect, meta


UNIX_TO_PG_DAYS = 10957                     # POSTGRES_EPOCH_JDATE - UNIX_EPOCH_JDATE


def arrow_groupby_session(lo_day=17532, hi_day=18262, ngroups_estimate=10_000_000.0):
    """WHERE d >= lo_day AND d < hi_day (Unix days) GROUP BY k -> count(*),
    sum(v1), min(v2), max(v2), sum(v2)."""
    from xb_producer import BoolOp
    vk, vv1, vv2, vd = Var(0, 1, "int8"), Var(0, 2, "int4"), Var(0, 3, "float8"), Var(0, 4, "date")
    sb = SessionBuilder(0, DEVTASK_PREAGG | DEVKIND_GPU)
    return sb.build(
        scan_quals=BoolOp("And", [Func("date_ge", [vd, Const("date", lo_day - UNIX_TO_PG_DAYS)], "bool"),
                                  Func("date_lt", [vd, Const("date", hi_day - UNIX_TO_PG_DAYS)], "bool")]),
        groupby_keys=[vk],
        aggs=[Agg("NROWS_ANY"), Agg("PSUM_INT", Func("int4_to_int8", [vv1], "int8")),
              Agg("PMIN_FP64", vv2), Agg("PMAX_FP64", vv2), Agg("PSUM_FP", vv2)],
        ngroups_estimate=float(ngroups_estimate))


def arrow_groupby(nrows=500_000_000, nkeys=10_000_000, seed_config=2, rows_per_chunk=2_500_000,
                  with_expect=True):
    """Arrow columnar high-cardinality pre-aggregation:
    k int8 U over nkeys, v1 int4 U[-1e6,1e6], v2 float8 lognormal(0,1),
    d Date32 U over 10 years from 2015-01-01, s dictionary text of 1000
    values (unreferenced: its buffers are not loaded, as Arrow_Fdw loads
    only referenced columns); WHERE d in [2018-01-01, 2020-01-01)
    GROUP BY k -> count(*), sum(v1), min(v2), max(v2), sum(v2).
    Returns (chunks, session, expect, meta)."""
    r = rng_for(seed_config, 0)
    d0 = 16436                                  # 2015-01-01 in Unix days
    lo_day, hi_day = 17532, 18262               # 2018-01-01, 2020-01-01
    typs = [("k", "int8"), ("v1", "int4"), ("v2", "float8"), ("d", "date"), ("s", "text")]
    session = arrow_groupby_session(lo_day, hi_day, float(min(nkeys, nrows)))
    chunks = []
    cols_all = {"k": [], "v1": [], "v2": [], "d": []}
    done = 0
    while done < nrows:
        n = min(rows_per_chunk, nrows - done)
        k = r.integers(0, nkeys, n, dtype=np.int64)
        v1 = r.integers(-1_000_000, 1_000_001, n, dtype=np.int32)
        v2 = r.lognormal(0.0, 1.0, n)
        d = r.integers(d0, d0 + 3652, n, dtype=np.int32)
        t = Table("t2", [Column(nm, ty) for nm, ty in typs], n)
        chunks.append(t.arrow_kds({
            "k": {"tag": 2, "bitwidth": 64, "values": k},
            "v1": {"tag": 2, "bitwidth": 32, "values": v1},
            "v2": {"tag": 3, "precision": 2, "values": v2},
            "d": {"tag": 8, "unit": 0, "values": d},
            "s": {"tag": 5},
        }))
        if with_expect:
            for nm, arr in (("k", k), ("v1", v1), ("v2", v2), ("d", d)):
                cols_all[nm].append(arr)
        done += n
    expect, meta = None, {"nitems_raw": nrows}
    if with_expect:
        k = np.concatenate(cols_all["k"]); v1 = np.concatenate(cols_all["v1"])
        v2 = np.concatenate(cols_all["v2"]); d = np.concatenate(cols_all["d"])
        m = (d >= lo_day) & (d < hi_day)
        km, v1m, v2m = k[m], v1[m].astype(np.int64), v2[m]
        order = np.argsort(km, kind="stable")     # stable: keeps row order per key
        ks, v1s, v2s = km[order], v1m[order], v2m[order]
        bounds = np.flatnonzero(np.diff(ks)) + 1
        starts = np.concatenate([[0], bounds])
        ends = np.concatenate([bounds, [len(ks)]])
        expect = {}
        for s_, e_ in zip(starts, ends):
            if e_ <= s_:
                continue
            vals = v2s[s_:e_]
            fsum = 0.0
            for x in vals:                        # row-ordered FP64 sum
                fsum += float(x)
            cnt = int(e_ - s_)
            expect[(int(ks[s_]),)] = [cnt, (cnt, int(v1s[s_:e_].sum())), (1, float(vals.min())),
                                      (1, float(vals.max())), (cnt, fsum)]
        meta.update({"nitems_in": int(m.sum()), "nitems_out": int(m.sum())})
    return chunks, session, expect, meta


def _validity(valid: np.ndarray) -> np.ndarray:
    """Arrow validity bitmap (bit i set: row i has a value, least significant
    bit first)"""
    return np.packbits(valid.astype(np.uint8), bitorder="little")


def arrow_nulls(nrows=200_000, nkeys=2_000, seed_config=37, rows_per_chunk=50_000, null_frac=0.1,
                short_rows=100):
    """The Arrow group-by's session over columns with NULLs: every
    referenced column carries a validity bitmap with null_frac of its rows
    NULL (k NULL: one group of its own; d NULL: the filter drops the row;
    v1 / v2 NULL: the aggregates skip it), and in every chunk the v2 values
    buffer ends short_rows rows before the chunk does, so those rows read as
    NULL (the readers' bound on values_length, KDS_ARROW_REF_SIMPLE_DATUM,
    xpu_common.h:1557-1574; the reference asserts that a row marked valid has
    a value, xpu_common.cu:273, so short_rows > 0 is for this library's
    readers and the oracle only).  Returns (chunks, session, expect, meta)."""
    r = rng_for(seed_config, 0)
    d0 = 16436
    lo_day, hi_day = 17532, 18262
    typs = [("k", "int8"), ("v1", "int4"), ("v2", "float8"), ("d", "date")]
    session = arrow_groupby_session(lo_day, hi_day, float(nkeys))
    chunks = []
    rows = {nm: [] for nm in ("k", "v1", "v2", "d", "kn", "v1n", "v2n", "dn")}
    done = 0
    while done < nrows:
        n = min(rows_per_chunk, nrows - done)
        k = r.integers(0, nkeys, n, dtype=np.int64)
        v1 = r.integers(-1_000_000, 1_000_001, n, dtype=np.int32)
        v2 = r.lognormal(0.0, 1.0, n)
        d = r.integers(d0, d0 + 3652, n, dtype=np.int32)
        nulls = {nm: r.random(n) < null_frac for nm in ("k", "v1", "v2", "d")}
        short = np.zeros(n, dtype=bool)
        short[max(0, n - short_rows):] = True
        t = Table("t2n", [Column(nm, ty) for nm, ty in typs], n)
        chunks.append(t.arrow_kds({
            "k": {"tag": 2, "bitwidth": 64, "values": k, "validity": _validity(~nulls["k"])},
            "v1": {"tag": 2, "bitwidth": 32, "values": v1, "validity": _validity(~nulls["v1"])},
            "v2": {"tag": 3, "precision": 2, "values": v2[:n - short_rows], "validity": _validity(~nulls["v2"])},
            "d": {"tag": 8, "unit": 0, "values": d, "validity": _validity(~nulls["d"])},
        }))
        for nm, arr in (("k", k), ("v1", v1), ("v2", v2), ("d", d)):
            rows[nm].append(arr)
        rows["kn"].append(nulls["k"])
        rows["v1n"].append(nulls["v1"])
        rows["v2n"].append(nulls["v2"] | short)
        rows["dn"].append(nulls["d"])
        done += n
    c = {nm: np.concatenate(v) for nm, v in rows.items()}
    m = ~c["dn"] & (c["d"] >= lo_day) & (c["d"] < hi_day)
    expect = {}
    for i in np.flatnonzero(m).tolist():        # row order: the FP64 sums are row-ordered
        key = (None,) if c["kn"][i] else (int(c["k"][i]),)
        g = expect.setdefault(key, [0, [0, 0], [0, None], [0, None], [0, 0.0]])
        g[0] += 1
        if not c["v1n"][i]:
            g[1][0] += 1
            g[1][1] += int(c["v1"][i])
        if not c["v2n"][i]:
            x = float(c["v2"][i])
            g[2] = [1, x if g[2][1] is None else min(g[2][1], x)]
            g[3] = [1, x if g[3][1] is None else max(g[3][1], x)]
            g[4][0] += 1
            g[4][1] += x
    expect = {k: [v[0], tuple(v[1]), tuple(v[2]), tuple(v[3]), tuple(v[4])] for k, v in expect.items()}
    meta = {"nitems_raw": nrows, "nitems_in": int(m.sum()), "nitems_out": int(m.sum())}
    return chunks, session, expect, meta


# ---------------------------------------------------------------------------
def scan_projection(nrows=200_000, seed_config=0, null_frac=0.05, a_limit=300, htup_margin=0):
    """The scan_groupby table and filter, rows projected into kds_dst:
    (id int8, a int4, b float8 with NULLs, c numeric, a * 2 + g int4).
    expect maps id -> (a, b or None, c unscaled, a * 2 + g)."""
    tbl, _, _, _, _ = scan_groupby(nrows=nrows, seed_config=seed_config, null_frac=null_frac,
                                   a_limit=a_limit)
    id_ = tbl.col("id").values
    a, g = tbl.col("a").values, tbl.col("g").values
    b, bnull = tbl.col("b").values, tbl.col("b").nulls
    typmod_c = numeric_typmod(12, 2)
    vid, va, vb, vc, vg = (Var(0, 1, "int8"), Var(0, 2, "int4"), Var(0, 3, "float8"),
                           Var(0, 4, "numeric", typmod_c), Var(0, 5, "int4"))
    sb = SessionBuilder(0, DEVTASK_SCAN | DEVKIND_GPU)
    session = sb.build(
        scan_quals=Func("int4lt", [va, Const("int4", a_limit)], "bool"),
        projection=[vid, va, vb, vc,
                    Func("int4pl", [Func("int4mul", [va, Const("int4", 2)], "int4"), vg], "int4")],
        htup_margin=htup_margin)
    m = a < a_limit
    expect = {}
    for i in np.flatnonzero(m):
        expect[int(id_[i])] = (int(a[i]), None if bnull[i] else float(b[i]), int(a[i]) * 2 + int(g[i]))
    meta = {"nitems_raw": nrows, "nitems_in": int(m.sum()), "nitems_out": int(m.sum())}
    return tbl, session, expect, meta


def join_projection(nfact=60_000, ndim1=3_000, ndim2=400, seed_config=1, flag_limit=3,
                    dim1_copies=1, miss_frac=0.0, key_stride=1):
    """The join_groupby tables and joins, rows projected into kds_dst:
    (fk1 int4, qty * price int8, region text, flag int2), one row per fact
    row and matching dim1 copy.  Returns (fact, session, kmrels, meta);
    meta["rows"] is the sorted list of expected value tuples."""
    fact, _, kmrels, _, meta = join_groupby(nfact=nfact, ndim1=ndim1, ndim2=ndim2,
                                             seed_config=seed_config, flag_limit=flag_limit,
                                             key_stride=key_stride, dim1_copies=dim1_copies,
                                             miss_frac=miss_frac, with_rows=True)
    f_fk1, f_fk2, f_qty, f_price = (Var(0, 1, "int4"), Var(0, 2, "int4"),
                                    Var(0, 3, "int4"), Var(0, 4, "int8"))
    d1_pk, d1_region = Var(1, 1, "int4"), Var(1, 2, "text")
    d2_pk, d2_flag = Var(2, 1, "int4"), Var(2, 2, "int2")
    sb = SessionBuilder(2, DEVTASK_JOIN | DEVKIND_GPU)
    session = sb.build(
        joins=[([f_fk1], [Func("int4eq", [f_fk1, d1_pk], "bool")], []),
               ([f_fk2], [Func("int4eq", [f_fk2, d2_pk], "bool")],
                [Func("int24lt", [d2_flag, Const("int4", flag_limit)], "bool")])],
        projection=[f_fk1, Func("int48mul", [f_qty, f_price], "int8"), d1_region, d2_flag])
    return fact, session, kmrels, meta


# ---------------------------------------------------------------------------
HEAP_ROW_BYTES = 68          # scan_groupby tuple + line pointer, in heap pages


def pinned_dim1_session(nslots=8192):
    """GpuScan of the join's dim1 (pk int4, region text) projecting its
    rows into a pinned inner buffer: KDS_FORMAT_HASH rows hashed by
    HashValue(pk), the inner hash of the fact-dim1 join."""
    pk, region = Var(0, 1, "int4"), Var(0, 2, "text")
    sb = SessionBuilder(0, DEVTASK_SCAN | DEVKIND_GPU)
    return sb.build(projection=[pk, region], projection_hash=[pk], proj_nslots=nslots)


def empty_hash_kds(table, length, nslots):
    """An empty KDS_FORMAT_HASH buffer of table's columns: length bytes,
    nslots zeroed hash slots, no rows."""
    head = table.kds_header("h", 0)
    buf = np.zeros(length, dtype=np.uint8)
    buf[:len(head)] = np.frombuffer(bytes(head), dtype=np.uint8)
    struct.pack_into("<QQ", buf, 0, length, 0)
    struct.pack_into("<I", buf, 40, nslots)
    return buf


def mixed_commands(ncmds=256, min_bytes=64 << 10, max_bytes=64 << 20, min_sel=0.001, max_sel=0.9,
                   max_groups=1_000_000, seed_config=3):
    """Chunk commands on the scan_groupby schema, each its own session and
    one KDS_FORMAT_BLOCK chunk: chunk bytes log-uniform in [min_bytes,
    max_bytes], selectivity of a < t uniform in [min_sel, max_sel], group
    count (domain of g) log-uniform in [1, max_groups].  Returns a list of
    dicts (chunk, session, truth, meta, params)."""
    r = rng_for(seed_config, 0)
    out = []
    for i in range(ncmds):
        nbytes = float(np.exp(r.uniform(np.log(min_bytes), np.log(max_bytes))))
        sel = float(r.uniform(min_sel, max_sel))
        groups = int(np.exp(r.uniform(0.0, np.log(max_groups))))
        nrows = max(1, int(nbytes // HEAP_ROW_BYTES))
        a_limit = max(1, int(round(sel * 1000)))
        tbl, sess, _, expect, meta = scan_groupby(nrows=nrows, seed_config=1000 + i, a_limit=a_limit,
                                                  ngroups=max(1, groups))
        chunks = tbl.block_chunks(pages_per_chunk=nrows // 60 + 2)   # >= 60 rows fill a page
        assert len(chunks) == 1
        chunk = chunks[0]
        truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
        out.append({"chunk": chunk, "session": sess, "truth": truth, "meta": meta,
                    "params": {"rows": nrows, "a_limit": a_limit, "groups": groups}})
    return out


def arrow_int2_bool(workdir, nrows=30_000, seed=33, null_frac=0.1, batch_rows=7_001):
    """An Arrow IPC file written into workdir (k int16, flag bool with NULLs,
    v int32, w int64; record batches of batch_rows rows, each batch's last
    bitmap byte partly used) read back by the chunk producer, and
    WHERE flag GROUP BY k -> count(*), sum(v::int8), min(w), max(w).
    Returns (chunks, session, expect, meta)."""
    import os
    import pyarrow as pa
    import xb_files as XF
    r = np.random.default_rng(seed)
    k = r.integers(-300, 300, nrows).astype(np.int16)
    flag = r.random(nrows) < 0.6
    fnull = r.random(nrows) < null_frac
    v = r.integers(-10**6, 10**6, nrows, dtype=np.int32)
    w = r.integers(-10**15, 10**15, nrows, dtype=np.int64)
    tbl = pa.table({"k": pa.array(k), "flag": pa.array(flag, mask=fnull), "v": pa.array(v),
                    "w": pa.array(w)})
    path = os.path.join(workdir, "int2_bool.arrow")
    with pa.OSFile(path, "wb") as sink:
        with pa.ipc.new_file(sink, tbl.schema) as wr:
            for b in tbl.to_batches(max_chunksize=batch_rows):
                wr.write_batch(b)
    chunks, tdef = XF.arrow_ipc_chunks(path)
    vk, vf, vv, vw = Var(0, 1, "int2"), Var(0, 2, "bool"), Var(0, 3, "int4"), Var(0, 4, "int8")
    session = SessionBuilder(0, DEVTASK_PREAGG | DEVKIND_GPU).build(
        scan_quals=vf,
        groupby_keys=[vk],
        aggs=[Agg("NROWS_ANY"), Agg("PSUM_INT", Func("int4_to_int8", [vv], "int8")),
              Agg("PMIN_INT64", vw), Agg("PMAX_INT64", vw)],
        ngroups_estimate=600.0)
    m = flag & ~fnull
    expect = {}
    for key in np.unique(k[m]).tolist():
        sel = m & (k == key)
        n = int(sel.sum())
        expect[(key,)] = [n, (n, int(v[sel].astype(np.int64).sum())), (1, int(w[sel].min())),
                          (1, int(w[sel].max()))]
    meta = {"nitems_raw": nrows, "nitems_in": int(m.sum()), "nitems_out": int(m.sum()),
            "types": [c.typ for c in tdef.columns]}
    return chunks, session, expect, meta

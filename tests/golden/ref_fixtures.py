"""
Golden vectors computed by PG-Strom's own functions, committed so that the
oracle's pin travels without the reference sources.

Run as a script where oracle/_ref/libref_xpu.so is built (oracle/Makefile
"ref": PG-Strom's expression library host-compiled from its sources, driven by
oracle/ref_harness.cpp):

    python tests/golden/ref_fixtures.py

It writes, next to this file:

* ref_scalars.json -- pg_hash_any (src/xpu_common.cu:2921) of seeded byte
  strings, and the reference's decode of numerics as xb_producer encodes
  them (__decimal_from_varlena, src/xpu_numeric.h:217);
* ref_pin_<case>.json -- per configuration, the row counters and every group
  (keys and partial states) that ExecLoadVarsOuterHeap / ExecLoadVarsOuterArrow,
  the quals, the hash joins and the aggregate functions of the reference
  compute over the chunks and bytecode that xb_configs produces, with the
  SHA-256 of those inputs so a drift of the generators is told apart from a
  drift of the oracle;
* ref_proj_<case>.json -- per projection configuration, the row counters,
  the number and SHA-256 of the tuples the reference forms, and the first
  few of them.

tests/test_golden_ref.py checks the C oracle against these files on any host.
TEST INFRASTRUCTURE ONLY.
"""
import hashlib
import json
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
for _sub in ("pg-strom_b200", os.path.join("pg-strom_b200", "producer"), "oracle"):
    _p = os.path.join(ROOT, _sub)
    if _p not in sys.path:
        sys.path.insert(0, _p)

import xb_configs as C  # noqa: E402
import xb_final as F  # noqa: E402

# small enough that the oracle finishes each in about a second and each file
# stays a few tens of KB
CASES = ("scan", "nogroup", "wide", "join", "long_varlena", "join_long_text", "arrow", "arrow_nulls",
         "filtered", "row_long_varlena", "arrow_int2_bool")

# projection sessions: rows formed into a KDS_FORMAT_ROW kds_dst by the
# reference's kern_estimate_minimal_tuple / kern_form_minimal_tuple
# (src/xpu_common.cu:1097-1300); the vectors keep the SHA-256 of the sorted
# tuple images (row id cut off) and the first few images in full
PROJ_CASES = ("scan_proj", "scan_proj_nulls", "join_proj", "join_proj_multi")
PROJ_SAMPLE = 8

HASH_LENGTHS = list(range(0, 48)) + [63, 64, 65, 100, 255, 1000]
NUMERIC_SCALES = (0, 2, 4)


def case_inputs(which):
    """(session, chunks, kmrels or None, meta) of one configuration."""
    if which == "scan":
        tbl, sess, km, _, meta = C.scan_groupby(nrows=60_000)
        chunks = tbl.block_chunks(pages_per_chunk=200)
    elif which == "nogroup":
        tbl, sess, km, _, meta = C.scan_nogroup(nrows=60_000)
        chunks = tbl.block_chunks(pages_per_chunk=200)
    elif which == "wide":
        # every partial-state form: count, count(x), int and float min/max,
        # float sum, numeric avg, stddev, covar
        tbl, sess, km, _, meta = C.wide_groupby(nrows=40_000, ngroups=300)
        chunks = tbl.block_chunks(pages_per_chunk=100)
    elif which == "join":
        tbl, sess, km, _, meta = C.join_groupby(nfact=60_000, ndim1=3000, ndim2=500)
        chunks = tbl.block_chunks(pages_per_chunk=200)
    elif which == "long_varlena":
        tbl, sess, km, _, meta = C.long_varlena_groupby(nrows=20_000)
        chunks = tbl.block_chunks(pages_per_chunk=100)
    elif which == "join_long_text":
        tbl, sess, km, _, meta = C.join_groupby(nfact=40_000, ndim1=3000, ndim2=500,
                                                regions=C.long_strings(40))
        chunks = tbl.block_chunks(pages_per_chunk=200)
    elif which == "arrow":
        chunks, sess, _, meta = C.arrow_groupby(nrows=30_000, nkeys=400, rows_per_chunk=12_000)
        km = None
    elif which == "arrow_nulls":
        # validity-bitmap NULLs only: the reference asserts that a row its
        # bitmap marks valid has a value (src/xpu_common.cu:273)
        chunks, sess, _, meta = C.arrow_nulls(nrows=30_000, nkeys=300, rows_per_chunk=10_000, short_rows=0)
        km = None
    elif which == "filtered":
        # line pointers partly LP_UNUSED / LP_DEAD / LP_REDIRECT
        chunks, sess, _, meta = C.scan_groupby_filtered(nrows=40_000, frac=0.2)
        km = None
    elif which == "row_long_varlena":
        # KDS_FORMAT_ROW outer chunks (kern_tupitems) of the long-varlena table
        tbl, sess, km, _, meta = C.long_varlena_groupby(nrows=12_000)
        chunks = tbl.row_chunks(rows_per_chunk=5_000)
    elif which == "arrow_int2_bool":
        # Arrow Int16 keys and a bit-packed Bool filter with NULLs, through an IPC file
        import tempfile
        with tempfile.TemporaryDirectory() as d:
            chunks, sess, _, meta = C.arrow_int2_bool(d)
        km = None
    elif which == "scan_proj":
        tbl, sess, _, meta = C.scan_projection(nrows=20_000)
        chunks, km = tbl.block_chunks(pages_per_chunk=64), None
    elif which == "scan_proj_nulls":
        tbl, sess, _, meta = C.scan_projection(nrows=12_000, null_frac=0.5, htup_margin=24)
        chunks, km = tbl.block_chunks(pages_per_chunk=64), None
    elif which == "join_proj":
        tbl, sess, km, meta = C.join_projection(nfact=20_000)
        chunks = tbl.block_chunks(pages_per_chunk=64)
    elif which == "join_proj_multi":
        # several dim1 rows per key and fact keys without a match
        tbl, sess, km, meta = C.join_projection(nfact=12_000, dim1_copies=3, miss_frac=0.2, key_stride=2)
        chunks = tbl.block_chunks(pages_per_chunk=64)
    else:
        raise ValueError(which)
    return sess, chunks, km, meta


def rows_digest(images):
    """SHA-256 of the sorted tuple images, each preceded by its length."""
    h = hashlib.sha256()
    for img in sorted(images):
        h.update(len(img).to_bytes(4, "little"))
        h.update(img)
    return h.hexdigest()


def input_digest(sess, chunks, km):
    h = hashlib.sha256()
    h.update(bytes(sess))
    for ch in chunks:
        h.update(np.ascontiguousarray(ch).tobytes())
    if km is not None:
        h.update(np.ascontiguousarray(km).tobytes())
    return h.hexdigest()


def hash_inputs():
    r = np.random.default_rng(11)
    return [r.integers(0, 256, n, dtype=np.uint8).tobytes() for n in HASH_LENGTHS]


def numeric_inputs():
    r = np.random.default_rng(12)
    vals = [0, 1, -1, 5, 10, 100, 9999, 10000, 123456, 999999, -999999, 1000000, 12300]
    vals += [int(v) for v in r.integers(-10**9, 10**9, 60)]
    return [(v, s) for s in NUMERIC_SCALES for v in vals]


def decode_groups(res, sess):
    """The harness's groups as {keys: states} in xb_final's decoded form:
    text keys without their 4-byte header, integers as Python ints, float
    states exact (the harness prints them with 17 significant digits)."""
    aggs = F.session_aggs(sess)
    stypes = F.slot_types(sess)
    keytypes = [stypes[a0] for (act, a0, _) in aggs if act == 101]
    out = {}
    for g in res["groups"]:
        keys = []
        for hexv, tc in zip(g["keys"], keytypes):
            if hexv is None:
                keys.append(None)
                continue
            b = bytes.fromhex(hexv)
            keys.append(b[4:] if tc == 11 else int.from_bytes(b, "little", signed=True))
        states = []
        for st, (action, _, typmod) in zip(g["states"], [a for a in aggs if a[0] != 101]):
            if action in (201, 202):
                states.append(st)
            elif action in (503, 603):
                states.append((st[0], float(st[1])))
            elif action in (304, 404):
                states.append((st[0], float(st[1]) if st[0] else None))
            elif action == 701:
                states.append((st[0], float(st[1]), float(st[2])))
            elif action == 801:
                states.append((st[0],) + tuple(float(v) for v in st[1:]))
            elif action in (504, 604):
                w = (((typmod - 4) & 0x7FF) ^ 1024) - 1024 if typmod >= 0 else 15
                states.append((st[0], int(st[1]), max(0, min(15, w))))
            else:
                states.append((st[0], int(st[1])))
        out[tuple(keys)] = states
    return out


def fixture_path(name):
    return os.path.join(HERE, name)


def load(name):
    with open(fixture_path(name)) as f:
        return json.load(f)


def generate():
    import ref_pin
    import xb_producer as P
    if not ref_pin.available():
        raise SystemExit("oracle/_ref/libref_xpu.so is not built (make -C oracle ref PGSTROM_SRC=...)")
    scal = {
        "hash_any": [[d.hex(), ref_pin.hash_any(d)] for d in hash_inputs()],
        "numeric": [],
    }
    for v, s in numeric_inputs():
        kind, w, iv = ref_pin.numeric_decode(P.encode_numeric(v, s))
        scal["numeric"].append([v, s, kind, w, str(iv)])
    with open(fixture_path("ref_scalars.json"), "w") as f:
        json.dump(scal, f, separators=(",", ":"))
    for which in CASES:
        sess, chunks, km, meta = case_inputs(which)
        res = ref_pin.run(sess, chunks, km)
        out = {
            "case": which,
            "inputs_sha256": input_digest(sess, chunks, km),
            "nitems_raw": res["nitems_raw"],
            "nitems_in": res["nitems_in"],
            "nitems_out": res["nitems_out"],
            "groups": res["groups"],
        }
        with open(fixture_path(f"ref_pin_{which}.json"), "w") as f:
            json.dump(out, f, separators=(",", ":"))
        print(f"{which}: {len(res['groups'])} groups, {res['nitems_raw']} rows")
    for which in PROJ_CASES:
        sess, chunks, km, meta = case_inputs(which)
        res = ref_pin.run(sess, chunks, km)
        images = sorted(bytes.fromhex(h) for h in res["rows"])
        out = {
            "case": which,
            "inputs_sha256": input_digest(sess, chunks, km),
            "nitems_raw": res["nitems_raw"],
            "nitems_in": res["nitems_in"],
            "nitems_out": res["nitems_out"],
            "nrows": len(images),
            "rows_sha256": rows_digest(images),
            "first_rows": [img.hex() for img in images[:PROJ_SAMPLE]],
        }
        with open(fixture_path(f"ref_proj_{which}.json"), "w") as f:
            json.dump(out, f, separators=(",", ":"))
        print(f"{which}: {len(images)} projected rows")


if __name__ == "__main__":
    generate()

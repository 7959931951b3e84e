"""The oracle against golden vectors that PG-Strom's own functions computed
(tests/golden/ref_fixtures.py, from the reference's expression library
host-compiled by oracle/Makefile "ref").  Unlike test_ref_pin.py this needs
neither the reference sources nor oracle/_ref: the vectors are committed.

Each configuration's inputs are regenerated from their seeds and must hash to
the digest recorded with the vectors; the oracle's groups must then equal the
reference's exactly (rtol=0: integer and numeric states bit-exact, float8
states to the last bit, as both sum in row order)."""
import os
import sys

import pytest

import xb_final as F
import xb_oracle as O
import xb_producer as P

sys.path.insert(0, os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden"))
import ref_fixtures as G  # noqa: E402


def test_hash_any_golden():
    vec = G.load("ref_scalars.json")["hash_any"]
    inputs = G.hash_inputs()
    assert len(vec) == len(inputs) == len(G.HASH_LENGTHS)
    for d, (hexd, want) in zip(inputs, vec):
        assert d.hex() == hexd
        assert P.hash_any(d) == want
        assert O.hash_bytes(d) == want


def test_numeric_encoding_golden():
    """xb_producer's numeric varlenas read back, by the reference's decoder,
    as the values they encode: kind 0 (finite) and value == v * 10^-scale."""
    vec = G.load("ref_scalars.json")["numeric"]
    assert [(v, s) for v, s, *_ in vec] == G.numeric_inputs()
    for v, scale, kind, w, iv in vec:
        iv = int(iv)
        assert kind == 0
        assert iv * 10 ** (scale - w if scale >= w else 0) == v * 10 ** (w - scale if w > scale else 0)


@pytest.mark.parametrize("which", G.CASES)
def test_oracle_matches_reference_golden(which):
    fx = G.load(f"ref_pin_{which}.json")
    sess, chunks, km, meta = G.case_inputs(which)
    assert G.input_digest(sess, chunks, km) == fx["inputs_sha256"], \
        "the generator's inputs drifted from those the vectors were made from: rerun tests/golden/ref_fixtures.py"
    assert fx["nitems_raw"] == meta["nitems_raw"]
    assert fx["nitems_in"] == meta["nitems_in"]
    assert fx["nitems_out"] == meta["nitems_out"]
    ref = G.decode_groups(fx, sess)
    assert len(ref) == len(fx["groups"])
    o = O.Oracle(sess, km)
    for ch in chunks:
        o.exec(ch)
    mine = F.decode_kds_final(o.final(), sess)
    st = o.stats()
    o.close()
    assert st["nitems_out"] == fx["nitems_out"]
    assert F.compare_groups(mine, ref, rtol=0.0) == []


@pytest.mark.parametrize("which", G.PROJ_CASES)
def test_oracle_projection_matches_reference_golden(which):
    """Projected rows: the oracle's tuple images (kern_tupitem, row id cut
    off) are, as a multiset, byte for byte those the reference's
    kern_form_minimal_tuple formed: same count, same SHA-256 of the sorted
    images, same first images."""
    fx = G.load(f"ref_proj_{which}.json")
    sess, chunks, km, meta = G.case_inputs(which)
    assert G.input_digest(sess, chunks, km) == fx["inputs_sha256"], \
        "the generator's inputs drifted from those the vectors were made from: rerun tests/golden/ref_fixtures.py"
    o = O.Oracle(sess, km)
    for ch in chunks:
        o.exec(ch)
    rows, _ = o.proj_rows()
    st = o.stats()
    o.close()
    assert (st["nitems_raw"], st["nitems_in"], st["nitems_out"]) == \
        (fx["nitems_raw"], fx["nitems_in"], fx["nitems_out"])
    assert len(rows) == fx["nrows"]
    assert [r.hex() for r in sorted(rows)[:G.PROJ_SAMPLE]] == fx["first_rows"]
    assert G.rows_digest(rows) == fx["rows_sha256"]

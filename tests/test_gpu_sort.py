"""GPU-Sort of the final groups on the GPU (SortKeys in the session,
applied by xpuB200Final): the groups come out in the order of the sort
keys (NULL placement and direction included), cut by LIMIT or filtered by
the window rank, and each kept group's states equal the generator's
truth.  The expected rows are the oracle's groups ordered by the restated
comparator (xb_final.order_groups)."""
import math

import pytest

import xb_configs as C
import xb_final as F
import xb_oracle as O
import xpu_b200
from test_gpusort import SORTS

pytestmark = pytest.mark.gpu


def _close(x, y):
    if x is None or y is None:
        return x is None and y is None
    if isinstance(x, float) or isinstance(y, float):
        return math.isclose(float(x), float(y), rel_tol=1e-9, abs_tol=1e-12)
    return x == y


def _check(got_rows, want, sess, keys):
    vals = [F.sort_key_values(r, sess, keys) for r in got_rows]
    assert len(vals) == len(want)
    for p in range(1, len(vals)):
        assert F._cmp_values(vals[p - 1], vals[p], keys) <= 0, (p, vals[p - 1], vals[p])
    for p, (v, w) in enumerate(zip(vals, [v for v, _ in want])):
        assert all(_close(a, b) for a, b in zip(v, w)), (p, v, w)
    assert sorted(k for k, _ in got_rows) == sorted(r[0] for _, r in want)


@pytest.fixture(scope="module")
def wide():
    tbl, sess, _, expect, meta = C.wide_groupby(nrows=400_000, ngroups=3000, seed_config=41)
    chunks = tbl.block_chunks(pages_per_chunk=512)
    o = O.Oracle(sess)
    for ch in chunks:
        o.exec(ch)
    rows = list(F.decode_kds_final(o.final(), sess).items())
    o.close()
    return chunks, rows, expect


@pytest.mark.parametrize("i", range(len(SORTS)))
def test_sorted_final_matches_restated_order(device, wide, i):
    chunks, orows, expect = wide
    sort = SORTS[i]
    sess = C.wide_groupby_session(sort=sort)
    s = xpu_b200.Session(device, sess)
    try:
        for ch in chunks:
            s.exec(ch)
        final, res = s.final()
    finally:
        s.close()
    got = F.decode_kds_final(final, sess)
    want = F.order_groups(orows, sess, sort["keys"], sort.get("window"), sort.get("limit", 0))
    assert res["final_nitems"] == len(want)
    _check(list(got.items()), want, sess, sort["keys"])
    assert F.compare_groups(got, {k: expect[k] for k in got}) == []


def test_sorted_join_groups_on_the_interpreter(device, monkeypatch):
    # 128-bit sums (sum(qty * price)) in descending order, first 10
    monkeypatch.setenv("XPU_B200_JIT", "0")
    fact, _, km, expect, meta = C.join_groupby(nfact=300_000, ndim1=5_000, ndim2=700, seed_config=42)
    sort = {"keys": [("PSUM_NUMERIC", 1, False, False)], "limit": 10}
    sess = C.join_groupby_session(sort=sort)
    s = xpu_b200.Session(device, sess, km, 2)
    try:
        for ch in fact.block_chunks(pages_per_chunk=300):
            s.exec(ch)
        final, _ = s.final()
    finally:
        s.close()
    got = list(F.decode_kds_final(final, sess).items())
    truth = sorted(expect.items(), key=lambda kv: -kv[1]["sum_amount"][1])[:10]
    assert [k for k, _ in got] == [k for k, _ in truth]
    assert [v[0] for _, v in got] == [tuple(t["sum_amount"]) for _, t in truth]


def test_sort_without_groups(device):
    tbl, sess0, _, _, _ = C.wide_groupby(nrows=5_000, a_limit=0, ngroups=10, seed_config=43)
    sess = C.wide_groupby_session(a_limit=0, ngroups=10, sort=SORTS[0])
    s = xpu_b200.Session(device, sess)
    try:
        for ch in tbl.block_chunks():
            s.exec(ch)
        final, res = s.final()
    finally:
        s.close()
    assert res["final_nitems"] == 0
    assert final is None or F.decode_kds_final(final, sess) == {}


@pytest.mark.parametrize("i", [1, 3, 6])
def test_sorted_final_many_groups(device, i):
    # 60,000 groups: the radix passes and scans span many 4096-element tiles
    tbl, _, _, expect, meta = C.wide_groupby(nrows=400_000, ngroups=60_000, seed_config=44)
    chunks = tbl.block_chunks(pages_per_chunk=512)
    sort = SORTS[i]
    sess = C.wide_groupby_session(ngroups=60_000, sort=sort)
    o = O.Oracle(sess)
    for ch in chunks:
        o.exec(ch)
    orows = list(F.decode_kds_final(o.final(), sess).items())
    o.close()
    s = xpu_b200.Session(device, sess)
    try:
        for ch in chunks:
            s.exec(ch)
        final, res = s.final()
    finally:
        s.close()
    got = F.decode_kds_final(final, sess)
    want = F.order_groups(orows, sess, sort["keys"], sort.get("window"), sort.get("limit", 0))
    assert res["final_nitems"] == len(want)
    _check(list(got.items()), want, sess, sort["keys"])
    assert F.compare_groups(got, {k: expect[k] for k in got}) == []

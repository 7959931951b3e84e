"""GPU-Sort of the final groups, host side: the SortKeys translation
(accepted key kinds, rejected ones with a message) and the restated
ordering (order_groups) against a direct sort of the generator's truth."""
import ctypes

import pytest

import xb_configs as C
import xb_final as F
import xb_oracle as O
import xpu_b200


def _translate(sess):
    L = ctypes.CDLL(xpu_b200.LIB_PATH)
    plan = ctypes.create_string_buffer(1 << 20)
    err = ctypes.create_string_buffer(1024)
    rc = L.xb_compile_session(bytes(sess), ctypes.c_size_t(len(sess)), ctypes.c_uint64(1 << 32), None, plan,
                              err, ctypes.c_size_t(1024))
    return rc, err.value.decode()


SORTS = [
    {"keys": [("PSUM_FP64", 7, False, False)], "limit": 50},
    {"keys": [("VREF", 2, True, False), ("VREF", 11, False, False)]},
    {"keys": [("PVARIANCE_SAMP", 9, True, True), ("VREF", 11, True, False)], "limit": 200},
    {"keys": [("VREF", 1, True, False), ("PMINMAX_FP64", 6, False, False)], "window": ("r", 1, 1, 2)},
    {"keys": [("VREF", 1, True, False), ("PMINMAX_FP64", 5, True, False)], "window": ("d", 1, 1, 1)},
    {"keys": [("PCOVAR_CORR", 10, False, False), ("PAVG_NUMERIC", 8, True, False)], "limit": 100},
    {"keys": [("PMINMAX_INT64", 3, True, False), ("PMINMAX_INT64", 4, False, False), ("VREF", 11, True, False)]},
]


@pytest.mark.parametrize("sort", SORTS)
def test_sort_keys_translate(sort):
    rc, msg = _translate(C.wide_groupby_session(sort=sort))
    assert rc == 0, msg


def test_sort_on_text_key_is_rejected():
    rc, msg = _translate(C.join_groupby_session(sort={"keys": [("VREF", 3, True, False)]}))
    assert rc != 0 and "not supported" in msg


def test_order_groups_matches_truth():
    # the oracle's groups ordered by sum(b) desc, cut at 40, are the 40
    # groups of largest sum(b) in the generator's truth
    tbl, sess, _, expect, meta = C.wide_groupby(nrows=60_000, ngroups=500)
    o = O.Oracle(sess)
    for ch in tbl.block_chunks(pages_per_chunk=100):
        o.exec(ch)
    rows = list(F.decode_kds_final(o.final(), sess).items())
    o.close()
    keys = [("PSUM_FP64", 7, False, False)]
    got = F.order_groups(rows, sess, keys, limit=40)
    want = sorted(expect, key=lambda k: -float(expect[k][6][1]))[:40]
    assert [r[0] for _, r in got] == want
    # window: the first row_number within each count(*) partition
    got = F.order_groups(rows, sess, [("VREF", 1, True, False), ("PMINMAX_FP64", 6, False, False)],
                         window=("n", 1, 1, 1))
    best = {}
    for k, v in expect.items():
        c = v[0]
        if c not in best or v[5][1] > expect[best[c]][5][1]:
            best[c] = k
    assert sorted(r[0] for _, r in got) == sorted(best.values())

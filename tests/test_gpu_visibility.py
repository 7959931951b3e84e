"""Heap pages that are not all-visible: PG-Strom's relscan.c sets the line
pointers of tuples the snapshot cannot see to LP_UNUSED before the pages
reach the GPU (src/relscan.c:462-494), and HOT pruning leaves LP_DEAD and
LP_REDIRECT items.  Only LP_NORMAL items are rows: both device kernels must
count and aggregate exactly the rows the oracle and the generator's truth
keep (integer and numeric states bit-exact, float8 sums within 1e-12
relative of the row-ordered sum)."""
import pytest

import xb_configs as C
import xb_final as F
from test_gpu_parity import kernel, run_gpu, run_oracle  # noqa: F401  (fixture)

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nrows,ppc,frac", [(30_000, 64, 0.2), (300_000, 1000, 0.05)])
def test_invalidated_line_pointers_parity(device, kernel, nrows, ppc, frac):
    chunks, sess, expect, meta = C.scan_groupby_filtered(nrows=nrows, frac=frac, pages_per_chunk=ppc)
    final, st, res = run_gpu(device, sess, chunks, kernel=kernel)
    assert st["nitems_raw"] == meta["nitems_raw"]
    assert st["nitems_in"] == meta["nitems_in"]
    got = F.decode_kds_final(final, sess)
    ofinal, _ = run_oracle(sess, chunks)
    assert F.compare_groups(got, F.decode_kds_final(ofinal, sess)) == []
    truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
    assert F.compare_groups(got, truth) == []

"""Inner relations resident across sessions (join_inner_handle): a session
with a handle builds the dimension indexes once; later sessions with the
same handle and build inputs use them as they are ("hit"), sessions whose
build differs (another hoisted inner qual constant) build their own, and
every result equals the generator's truth.  Unreferenced builds leave when
the budget shrinks."""
import pytest

import xb_configs as C
import xb_final as F
import xpu_b200

pytestmark = pytest.mark.gpu


def _run(device, sess, km, chunks, expect):
    s = xpu_b200.Session(device, sess, km, 2)
    try:
        state = s.info()["inner_cache"]
        for ch in chunks:
            s.exec(ch)
        final, _ = s.final()
    finally:
        s.close()
    truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    assert F.compare_groups(F.decode_kds_final(final, sess), truth) == []
    return state


@pytest.mark.parametrize("jit", ["1", "0"])
def test_inner_relations_resident_across_sessions(device, monkeypatch, jit):
    monkeypatch.setenv("XPU_B200_JIT", jit)
    handle = 0x100 + int(jit)
    fact, _, km, expect3, meta = C.join_groupby(nfact=200_000, ndim1=20_000, ndim2=700, seed_config=51)
    _, _, _, expect2, _ = C.join_groupby(nfact=200_000, ndim1=20_000, ndim2=700, seed_config=51, flag_limit=2)
    chunks = fact.block_chunks(pages_per_chunk=200)
    device.inner_cache(16 << 30)
    s3 = C.join_groupby_session(flag_limit=3, inner_handle=handle)
    assert _run(device, s3, km, chunks, expect3) == "built"
    assert device.inner_cache() > 0
    assert _run(device, s3, km, chunks, expect3) == "hit"
    # dim2's hoisted qual has another constant: another build
    s2 = C.join_groupby_session(flag_limit=2, inner_handle=handle)
    assert _run(device, s2, km, chunks, expect2) == "built"
    assert _run(device, s2, km, chunks, expect2) == "hit"
    # two sessions at once share one build
    a = xpu_b200.Session(device, s3, km, 2)
    b = xpu_b200.Session(device, s3, km, 2)
    try:
        assert a.info()["inner_cache"] == "hit" and b.info()["inner_cache"] == "hit"
        for ch in chunks:
            a.exec(ch)
            b.exec(ch)
        fa, _ = a.final()
        fb, _ = b.final()
        assert F.decode_kds_final(fa, s3) == F.decode_kds_final(fb, s3)
    finally:
        a.close()
        b.close()
    # no handle: nothing cached
    s0 = C.join_groupby_session(flag_limit=3)
    assert _run(device, s0, km, chunks, expect3) == "none"
    # a zero budget drops every unreferenced build
    assert device.inner_cache(0) == 0
    assert _run(device, s3, km, chunks, expect3) == "built"
    device.inner_cache(16 << 30)

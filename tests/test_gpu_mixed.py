"""Mixed batches: chunk commands of many sessions in one persistent launch
(xpuB200MixCreate / xpuB200MixExec, replayed from a captured CUDA graph).
Every command's groups must equal its generator's ground truth (integer and
numeric states exact, float8 sums within 1e-12 of the row-ordered FP64
sum), be the same as when the command runs alone, and be unaffected by the
other commands of the launch."""
import pytest

import xb_configs as C
import xb_final as F
import xb_oracle as O
import xpu_b200

pytestmark = pytest.mark.gpu


def _open_all(device, cmds):
    sessions, bases, dptrs = [], [], []
    for c in cmds:
        sessions.append(xpu_b200.Session(device, c["session"]))
        base, p = device.upload(c["chunk"])
        bases.append(base)
        dptrs.append(p)
    return sessions, bases, dptrs


def _close_all(device, sessions, bases):
    for s in sessions:
        s.close()
    for b in bases:
        device.free(b)


@pytest.fixture(params=["jit", "vm"])
def kernel(request, monkeypatch):
    monkeypatch.setenv("XPU_B200_JIT", "1" if request.param == "jit" else "0")
    return request.param


def test_mixed_batch_matches_truth_and_oracle(device, kernel):
    cmds = C.mixed_commands(ncmds=96, max_bytes=4 << 20, max_groups=100_000)
    sessions, bases, dptrs = _open_all(device, cmds)
    mix = xpu_b200.Mix(device, sessions, dptrs)
    try:
        info = mix.info()
        assert info["items"] >= len(cmds)
        # one plan shape: one persistent launch, specialised unless disabled
        assert info["launches"] == 1
        assert info["specialised"] == (len(cmds) if kernel == "jit" else 0)
        out = mix.exec()
        for i, ((res, err), c, s) in enumerate(zip(out, cmds, sessions)):
            assert err is None, f"command {i}: {err}"
            assert res["nitems_raw"] == c["meta"]["nitems_raw"], i
            assert res["nitems_in"] == c["meta"]["nitems_in"], i
            final, fres = s.final()
            got = F.decode_kds_final(final, c["session"]) if final is not None else {}
            assert F.compare_groups(got, c["truth"]) == [], f"command {i} {c['params']}"
            assert fres["final_nitems"] == len(c["truth"])
        # the oracle agrees on a few of them
        for c in cmds[:6]:
            o = O.Oracle(c["session"])
            o.exec(c["chunk"])
            ofinal = o.final()
            o.close()
            assert F.compare_groups(F.decode_kds_final(ofinal, c["session"]), c["truth"]) == []
    finally:
        mix.close()
        _close_all(device, sessions, bases)


def test_mixed_batch_same_as_alone(device):
    cmds = C.mixed_commands(ncmds=24, max_bytes=2 << 20, max_groups=20_000, seed_config=5)
    sessions, bases, dptrs = _open_all(device, cmds)
    alone_sessions = [xpu_b200.Session(device, c["session"]) for c in cmds]
    mix = xpu_b200.Mix(device, sessions, dptrs)
    try:
        assert all(err is None for _, err in mix.exec())
        for c, s_mix, s_alone, p in zip(cmds, sessions, alone_sessions, dptrs):
            s_alone.exec(p, on_device=True)
            a, _ = s_alone.final()
            m, _ = s_mix.final()
            ga = F.decode_kds_final(a, c["session"]) if a is not None else {}
            gm = F.decode_kds_final(m, c["session"]) if m is not None else {}
            assert F.compare_groups(gm, ga) == []
    finally:
        mix.close()
        for s in alone_sessions:
            s.close()
        _close_all(device, sessions, bases)


def test_mixed_batch_several_chunks_of_one_session(device):
    # three chunks of one table share one session (and its group table)
    # next to other sessions' commands
    tbl, sess, _, expect, _ = C.scan_groupby(nrows=90_000, seed_config=7, ngroups=300)
    chunks = tbl.block_chunks(pages_per_chunk=300)
    assert len(chunks) >= 3
    others = C.mixed_commands(ncmds=8, max_bytes=1 << 20, max_groups=5_000, seed_config=6)
    s_main = xpu_b200.Session(device, sess)
    o_sessions, o_bases, o_dptrs = _open_all(device, others)
    bases, dptrs = [], []
    for ch in chunks:
        b, p = device.upload(ch)
        bases.append(b)
        dptrs.append(p)
    mix = xpu_b200.Mix(device, [s_main] * len(chunks) + o_sessions, dptrs + o_dptrs)
    try:
        assert all(err is None for _, err in mix.exec())
        final, _ = s_main.final()
        truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
        assert F.compare_groups(F.decode_kds_final(final, sess), truth) == []
        for c, s in zip(others, o_sessions):
            f, _ = s.final()
            got = F.decode_kds_final(f, c["session"]) if f is not None else {}
            assert F.compare_groups(got, c["truth"]) == []
    finally:
        mix.close()
        s_main.close()
        for b in bases:
            device.free(b)
        _close_all(device, o_sessions, o_bases)


def test_mixed_batch_of_two_plan_shapes(device):
    # join commands and scan commands: one persistent launch per kernel,
    # running concurrently inside the replayed graph
    fact, jsess, km, expect, _ = C.join_groupby(nfact=200_000, ndim1=20_000, ndim2=2_000)
    jchunks = fact.block_chunks(pages_per_chunk=400)
    scans = C.mixed_commands(ncmds=10, max_bytes=1 << 20, max_groups=5_000, seed_config=8)
    js = xpu_b200.Session(device, jsess, km, 2)
    s_sessions, s_bases, s_dptrs = _open_all(device, scans)
    j_bases, j_dptrs = [], []
    for ch in jchunks:
        b, p = device.upload(ch)
        j_bases.append(b)
        j_dptrs.append(p)
    mix = xpu_b200.Mix(device, [js] * len(jchunks) + s_sessions, j_dptrs + s_dptrs)
    try:
        assert mix.info()["launches"] == 2
        assert all(err is None for _, err in mix.exec())
        jf, _ = js.final()
        truth = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
        assert F.compare_groups(F.decode_kds_final(jf, jsess), truth) == []
        for c, s in zip(scans, s_sessions):
            f, _ = s.final()
            got = F.decode_kds_final(f, c["session"]) if f is not None else {}
            assert F.compare_groups(got, c["truth"]) == []
    finally:
        mix.close()
        js.close()
        for b in j_bases:
            device.free(b)
        _close_all(device, s_sessions, s_bases)

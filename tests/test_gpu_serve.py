"""Serving form: chunk commands of many sessions submitted asynchronously
(xpuB200Submit / xpuB200Poll) and batched by the device scheduler.  Each
command's result must be the same as when it runs alone, whatever else is
in flight: integer and numeric states exact, float8 sums within 1e-12 of
the row-ordered FP64 sum."""
import numpy as np
import pytest

import xb_configs as C
import xb_final as F
import xpu_b200

pytestmark = pytest.mark.gpu


def _finals(sessions, cmds):
    out = []
    for s, c in zip(sessions, cmds):
        f, _ = s.final()
        out.append(F.decode_kds_final(f, c["session"]) if f is not None else {})
    return out


@pytest.mark.parametrize("on_device", [False, True])
def test_served_commands_match_truth(device, on_device):
    cmds = C.mixed_commands(ncmds=64, max_bytes=4 << 20, max_groups=50_000, seed_config=11)
    sessions = [xpu_b200.Session(device, c["session"]) for c in cmds]
    bases, tickets = [], []
    try:
        for c, s in zip(cmds, sessions):
            if on_device:
                base, p = device.upload(c["chunk"])
                bases.append(base)
                tickets.append(device.submit(s, p, on_device=True))
            else:
                tickets.append(device.submit(s, c["chunk"]))
        for t, c in zip(tickets, cmds):
            r = device.poll(t)
            assert r["nitems_raw"] == c["meta"]["nitems_raw"]
            assert r["nitems_in"] == c["meta"]["nitems_in"]
        with pytest.raises(xpu_b200.XpuB200Error, match="unknown ticket"):
            device.poll(tickets[0])                  # reported done once
        for got, c in zip(_finals(sessions, cmds), cmds):
            assert F.compare_groups(got, c["truth"]) == [], c["params"]
    finally:
        for s in sessions:
            s.close()
        for b in bases:
            device.free(b)


def test_served_same_as_alone_with_large_commands(device):
    # large join commands (run alone on their specialised kernel) and small
    # scan commands (mixed launches) in flight together; a tight admission
    # budget makes later commands wait for memory
    fact, jsess, km, expect, meta = C.join_groupby(nfact=400_000, ndim1=20_000, ndim2=2_000)
    jchunks = fact.block_chunks(pages_per_chunk=600)
    small = C.mixed_commands(ncmds=40, max_bytes=2 << 20, max_groups=20_000, seed_config=12)
    device.serve_config(admit_bytes=24 << 20, alone_units=256)
    js = xpu_b200.Session(device, jsess, km, 2)
    ss = [xpu_b200.Session(device, c["session"]) for c in small]
    try:
        tickets = []
        order = list(range(len(jchunks) + len(small)))
        np.random.default_rng(3).shuffle(order)
        for k in order:
            if k < len(jchunks):
                tickets.append((device.submit(js, jchunks[k]), 2))
            else:
                c = small[k - len(jchunks)]
                tickets.append((device.submit(ss[k - len(jchunks)], c["chunk"]), 0))
        for t, nrels in tickets:
            device.poll(t, nrels=nrels)
        jf, _ = js.final()
        truth = {kk: [v["sum_amount"], v["nrows"]] for kk, v in expect.items()}
        assert F.compare_groups(F.decode_kds_final(jf, jsess), truth) == []
        # the join's plan shape may still be building: its commands ran on
        # the interpreter until then, on its specialised kernel after
        assert set(js.info()["kernels"].values()) <= {"jit", "vm"}
        for got, c in zip(_finals(ss, small), small):
            alone = xpu_b200.Session(device, c["session"])
            alone.exec(c["chunk"])
            af, _ = alone.final()
            alone.close()
            want = F.decode_kds_final(af, c["session"]) if af is not None else {}
            assert F.compare_groups(got, want) == []
            assert F.compare_groups(got, c["truth"]) == []
    finally:
        device.serve_config(admit_bytes=xpu_b200.ADMIT_FREE_HBM, alone_units=256)
        js.close()
        for s in ss:
            s.close()


def test_poll_without_wait_and_final_drains(device):
    cmds = C.mixed_commands(ncmds=12, max_bytes=1 << 20, max_groups=1_000, seed_config=13)
    sessions = [xpu_b200.Session(device, c["session"]) for c in cmds]
    try:
        tickets = [device.submit(s, c["chunk"]) for s, c in zip(sessions, cmds)]
        r = device.poll(tickets[-1], wait=False)
        assert r is None or r["nitems_raw"] == cmds[-1]["meta"]["nitems_raw"]
        # Final waits for the session's own submitted commands
        for got, c in zip(_finals(sessions, cmds), cmds):
            assert F.compare_groups(got, c["truth"]) == []
        for t in tickets:
            try:
                device.poll(t)
            except xpu_b200.XpuB200Error as e:   # already reported by the wait=False poll
                assert "unknown ticket" in str(e) and t == tickets[-1]
    finally:
        for s in sessions:
            s.close()


def _rare_shape_session(variant=0, ngroups=64):
    """A GROUP BY whose aggregate list no other test uses (variant adds
    count(*) columns), so that no specialised kernel exists for its plan
    shape when it is first served."""
    from xb_producer import Agg, Const, Func, SessionBuilder, Var
    va, vb, vg = Var(0, 2, "int4"), Var(0, 3, "float8"), Var(0, 5, "int4")
    return SessionBuilder(0, C.DEVTASK_PREAGG | C.DEVKIND_GPU).build(
        scan_quals=Func("int4lt", [va, Const("int4", 700)], "bool"),
        groupby_keys=[vg],
        aggs=[Agg("NROWS_ANY"), Agg("PMAX_INT32", va), Agg("PMIN_INT32", va), Agg("NROWS_COND", vb),
              Agg("PSUM_INT", Func("int4_to_int8", [va], "int8")), Agg("PMAX_FP64", vb)] +
             [Agg("NROWS_ANY")] * (1 + variant),
        ngroups_estimate=float(ngroups))


@pytest.mark.parametrize("alone", [True, False])
def test_new_plan_shape_served_while_its_kernel_builds(device, alone):
    """A served command of a plan shape without a kernel runs at once on
    the interpreting kernel while the specialised kernel builds on a
    background thread (NVRTC takes seconds); commands after the build run
    on the specialised kernel.  Every result equals the oracle's."""
    import time
    import xb_oracle as O
    tbl, _, _, _, _ = C.scan_groupby(nrows=300_000, seed_config=90 if alone else 91)
    sess = _rare_shape_session(variant=0 if alone else 1)
    # alone: commands of >= 256 heap pages run alone; else small ones, mixed
    chunks = tbl.block_chunks(pages_per_chunk=400 if alone else 60)
    device.serve_config(admit_bytes=xpu_b200.ADMIT_FREE_HBM, alone_units=256)
    s = xpu_b200.Session(device, sess)
    try:
        t0 = time.perf_counter()
        device.poll(device.submit(s, chunks[0]))
        first_s = time.perf_counter() - t0
        assert s.info()["kernels"] == {"b": "vm"}, s.info()
        used = 1
        deadline = time.perf_counter() + 120.0
        while time.perf_counter() < deadline:
            device.poll(device.submit(s, chunks[used % len(chunks)]))
            used += 1
            if s.info()["kernels"] == {"b": "jit"}:
                break
            time.sleep(0.2)
        assert s.info()["kernels"] == {"b": "jit"}, s.info()
        # the first command did not wait for the build
        assert first_s < s.info()["jit_compile_ms"] / 1000.0 or first_s < 1.0, (first_s, s.info())
        final, _ = s.final()
    finally:
        s.close()
    o = O.Oracle(sess)
    for i in range(used):
        o.exec(chunks[i % len(chunks)])
    want = F.decode_kds_final(o.final(), sess)
    o.close()
    assert F.compare_groups(F.decode_kds_final(final, sess), want) == []

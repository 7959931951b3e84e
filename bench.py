"""
Benchmark of the B200 scan / hash-join / pre-aggregation executor.

Workload (N=1): the two-way hash join + GROUP BY over heap pages -- a
100M-row fact table (fk1 uniform into dim1 of 200k rows, fk2 bounded
Zipf(1.1) into dim2 of 10k rows, qty, price) in 64 MB KDS_FORMAT_BLOCK
chunks, joined with dim1 (region text) and dim2 (flag < 3 as a pushed-down
join qual), GROUP BY region -> sum(qty*price), count(*).  Synthetic seeded
data with the configuration's shapes and distributions.

  value   rows/s with the chunks resident in HBM: one step = one pass of
          the executor over all chunks (one persistent launch), timed with
          CUDA events on the session stream;
  e2e     the same query end to end through the C ABI from pinned host
          memory: OpenSession (inner upload + index build), one ExecTask per
          chunk (host->device copy inside), Final (kds_final read back),
          CloseSession -- every step;
  roofline  the executor kernel against the measured HBM copy bandwidth;
  cpu_baseline  the reference's own expression library (host-compiled) or
          the C oracle, multi-threaded over a bounded sample, rank 0, N=1.

Multi-GPU (torchrun): weak scaling, every rank processes its own 100M-row
shard with no data-path collective; time = max over ranks.
"""
import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import threading
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
for sub in ("pg-strom_b200", os.path.join("pg-strom_b200", "producer"), "oracle"):
    sys.path.insert(0, os.path.join(ROOT, sub))

import numpy as np

METRIC = "scan+join+preagg rows/s"
UNIT = "rows/s"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--rows", type=int, default=100_000_000)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-seconds", type=float, default=12.0)
    ap.add_argument("--workload", default="join_groupby",
                    choices=["join_groupby", "scan_groupby", "arrow_groupby", "mixed", "served"],
                    help="join_groupby: the headline line; scan_groupby / arrow_groupby: the plain "
                         "scan and the Arrow high-cardinality configurations (--rows, --keys); mixed: "
                         "256 batched chunk commands; served: Poisson-arrival query mix through the "
                         "serving scheduler")
    ap.add_argument("--no-tune", dest="tune", action="store_false",
                    help="keep the default launch shape (no xpuB200BatchTune before timing)")
    ap.add_argument("--final-merge", default="gather", choices=["gather", "exchange"],
                    help="N>1: merge every rank's kds_final on rank 0 (gather), or split the groups "
                         "by hash across the ranks (exchange: all-to-all, each rank merges its share)")
    ap.add_argument("--keys", type=int, default=10_000_000)
    ap.add_argument("--requests", type=int, default=400)
    ap.add_argument("--qps", type=float, default=200.0)
    ap.add_argument("--served-arrow-rows", type=int, default=500_000_000,
                    help="served: rows of the Arrow template's table (queries take 1M..all of it)")
    ap.add_argument("--no-served-leg", dest="served_leg", action="store_false",
                    help="headline line: skip the short served-mix measurement")
    ap.add_argument("--no-reference-gpu", dest="reference_gpu", action="store_false",
                    help="skip the reference's own kernel (built for sm_100a) on the same GPU")
    ap.add_argument("--no-configs", dest="configs", action="store_false",
                    help="headline line: skip the C0 / C2 / C3 configuration runs")
    return ap.parse_args()


def dist_setup(n):
    rank, world = int(os.environ.get("RANK", "0")), int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import torch
        import torch.distributed as dist
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    return rank, world, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def _reduce(x, world, op):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=op)
    return float(t.item())


def max_over_ranks(x, world):
    """Step time of the job = the slowest rank's device time."""
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.MAX if world > 1 else None)


def sum_over_ranks(x, world):
    import torch.distributed as dist
    return _reduce(x, world, dist.ReduceOp.SUM if world > 1 else None)


def gather_finals(final, rank, world):
    """Every rank's kds_final (uint8 array or None) collected on rank 0 in
    rank order, as the GPU service collects one kds_final per GPU before
    merging them (gpu_service.c:5442-5518); None on the other ranks."""
    import numpy as np
    import torch.distributed as dist
    if world == 1:
        return [final]
    out = [None] * world if rank == 0 else None
    payload = None if final is None else memoryview(final).tobytes()
    dist.gather_object(payload, out, dst=0)
    if rank != 0:
        return None
    return [None if b is None else np.frombuffer(b, dtype=np.uint8).copy() for b in out]


def _tune(batch, args):
    """The launch shape the timed passes use: tuned on the batch itself
    (xpuB200BatchTune, before any pass counts) unless --no-tune."""
    if not args.tune:
        return {"tuned": False}
    rep = batch.tune()
    return {"tuned": True, "ctas_per_sm": rep["best"]["ctas_per_sm"], "sm_groups": rep["best"]["sm_groups"],
            "default_sm_groups": rep["default_sm_groups"],
            "measured_ms": {f'{c["ctas_per_sm"]}/{c["sm_groups"]}': round(c["ms"], 4) for c in rep["candidates"]}}


def shard_seed(rank):
    """Weak scaling: every rank generates and owns a distinct fact shard."""
    return 1 + 16 * rank


class ClockSampler:
    """SM clock and clock-event (throttle) reasons sampled during the timed
    region: NVML polled every 2 ms from a thread (the timed region of a step
    is tens of milliseconds), else nvidia-smi at its 200 ms floor.  Reads
    only; changes no GPU setting."""
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clocks-event reason bits
    BITS = {"sw_power_cap": 0x4, "hw_slowdown": 0x8, "sw_thermal_slowdown": 0x20,
            "hw_thermal_slowdown": 0x40}

    def __init__(self, gpu_index):
        vis = os.environ.get("CUDA_VISIBLE_DEVICES", "")
        ids = [x.strip() for x in vis.split(",") if x.strip()]
        self.gpu = int(ids[gpu_index]) if gpu_index < len(ids) and ids[gpu_index].isdigit() else gpu_index
        self.proc = None
        self.lines = []
        self.samples = []
        self.nvml = None
        self.stop_ev = threading.Event()

    def start(self):
        try:
            import pynvml
            pynvml.nvmlInit()
            h = pynvml.nvmlDeviceGetHandleByIndex(self.gpu)
            reasons = getattr(pynvml, "nvmlDeviceGetCurrentClocksEventReasons", None) or \
                pynvml.nvmlDeviceGetCurrentClocksThrottleReasons
            self.nvml = (pynvml, h, reasons)
            self.smax = pynvml.nvmlDeviceGetMaxClockInfo(h, pynvml.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._poll, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.nvml = None
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.FIELDS,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None

    def _poll(self):
        pynvml, h, reasons = self.nvml
        while not self.stop_ev.is_set():
            try:
                self.samples.append((pynvml.nvmlDeviceGetClockInfo(h, pynvml.NVML_CLOCK_SM), reasons(h)))
            except Exception:
                pass
            time.sleep(0.002)

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.nvml:
            self.stop_ev.set()
            self.thread.join(timeout=5)
            sm = [c for c, _ in self.samples]
            reasons = sorted({nm for _, r in self.samples for nm, bit in self.BITS.items() if r & bit})
            return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": self.smax,
                    "samples": len(sm), "reasons": reasons, "source": "nvml 2 ms"}
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["clock sampling unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            parts = [p.strip() for p in ln.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None,
                "sm_max_mhz": max(smax) if smax else None,
                "samples": len(sm), "reasons": sorted(reasons), "source": "nvidia-smi 200 ms"}


def build_workload(nrows, rank):
    import xb_configs as C
    fact, sess, km, expect, meta = C.join_groupby(nfact=nrows, seed_config=shard_seed(rank))
    chunks = fact.block_chunks(pages_per_chunk=8190)
    meta["truth"] = {k: [v["sum_amount"], v["nrows"]] for k, v in expect.items()}
    return fact, sess, km, chunks, meta


# ------------------------------------------------------------------ CPU arms
def cpu_rows_per_sec(sess, km, chunks, seconds, threads, allow_ref=True):
    """Runs the reference's host-compiled functions (or, where oracle/_ref
    was not built, the C oracle) over chunks on 'threads' threads until
    'seconds' of wall time; rows/s.  The reference harness reads heap,
    Arrow and ROW chunks and counts rows without writing its groups out."""
    import ref_pin
    import xb_oracle as O
    use_ref = allow_ref and ref_pin.available()
    kind = "reference" if use_ref else "port"
    lock = threading.Lock()
    state = {"rows": 0, "next": 0}
    deadline = time.perf_counter() + seconds

    def worker():
        o = None if use_ref else O.Oracle(sess, km)
        while time.perf_counter() < deadline:
            with lock:
                i = state["next"] % len(chunks)
                state["next"] += 1
            ch = chunks[i]
            if use_ref:
                n = ref_pin.run_counts(sess, [ch], km)["nitems_raw"]
            else:
                before = o.stats()["nitems_raw"]
                o.exec(ch)
                n = o.stats()["nitems_raw"] - before
            with lock:
                state["rows"] += n
        if o is not None:
            o.close()

    t0 = time.perf_counter()
    ths = [threading.Thread(target=worker) for _ in range(threads)]
    for t in ths:
        t.start()
    for t in ths:
        t.join()
    el = time.perf_counter() - t0
    return state["rows"] / el, kind, state["rows"], el


def reference_gpu_leg(sess, km, chunks, rows, truth, steps=3, warmup=1, rtol=None):
    """PG-Strom's own device executor, kern_gpujoin_main, built for sm_100a
    from the reference sources and launched as its GPU service launches it
    (one task and one stream synchronisation per chunk), over its own
    device copies of the same chunks on the same GPU.  Its groups are
    checked against the truth; the timed passes reuse one session, as the
    timed batches of this repository's path do."""
    import ref_gpu
    import xb_final as F
    if not ref_gpu.available():
        return {"unavailable": "the reference's sm_100a build (oracle/_ref) is not present"}
    ref_gpu.open_device(0)
    ptrs = [ref_gpu.upload(c) for c in chunks]
    try:
        rs = ref_gpu.RefSession(sess, km)
        try:
            rs.exec(ptrs)
            final = rs.final()
            got = F.decode_kds_final(final, sess)
            errs = (F.compare_groups(got, truth) if rtol is None else F.compare_groups(got, truth, rtol=rtol)) \
                if truth else []
            for _ in range(warmup):
                rs.exec(ptrs)
            k0 = rs.info()["kernel_ms"]
            times = [rs.exec(ptrs) for _ in range(steps)]
            info = rs.info()
        finally:
            rs.close()
    finally:
        for p in ptrs:
            ref_gpu.free(p)
    ms = sum(times) / len(times)
    kms = (info["kernel_ms"] - k0) / steps
    return {"value": rows / (ms / 1000.0), "unit": UNIT, "ms_per_pass": ms,
            "kernel_ms_per_pass": kms, "kernel_value": rows / (kms / 1000.0),
            "kernel": "kern_gpujoin_main (PG-Strom sources, sm_100a, --maxrregcount=128)",
            "tasks_per_pass": len(chunks),
            "launch": {k: info[k] for k in ("grid", "block", "shmem", "prepfn_nbufs", "registers",
                                            "stack_limit")},
            "includes": "ms_per_pass: every chunk's launch and the stream synchronisation after it, as the "
                        "reference's GPU service runs its tasks; kernel_ms_per_pass: the launches alone",
            "parity": {"groups_equal_truth": errs == [], "errors": errs[:3]}}


CONFIG_RUNS = [
    ("C0 scan_groupby 4M heap rows",
     ["--workload", "scan_groupby", "--rows", "4000000", "--steps", "10", "--warmup", "3", "--cpu-seconds", "4"]),
    ("C2 arrow_groupby 500M rows / 10M keys",
     ["--workload", "arrow_groupby", "--rows", "500000000", "--steps", "5", "--warmup", "3", "--cpu-seconds", "0"]),
    ("C3 mixed: 256 batched chunk commands",
     ["--workload", "mixed", "--steps", "10", "--warmup", "3"]),
]


def config_lines(timeout_s=240):
    """The other configurations of the benchmark, each in a process of its
    own after every measurement of the headline (one at a time, so they
    share the GPU with nothing): a short summary of each line."""
    out = {}
    for name, argv in CONFIG_RUNS:
        t0 = time.time()
        try:
            p = subprocess.run([sys.executable, os.path.abspath(__file__)] + argv, capture_output=True,
                               text=True, timeout=timeout_s)
            lines = [l for l in p.stdout.splitlines() if l.startswith("{")]
            if p.returncode != 0 or not lines:
                out[name] = {"error": (p.stderr or "no output").strip().splitlines()[-1][:300]}
                continue
            d = json.loads(lines[-1])
        except Exception as e:
            out[name] = {"error": f"{type(e).__name__}: {e}"[:300]}
            continue
        summ = {"metric": d.get("metric"), "value": d.get("value"), "unit": d.get("unit"),
                "ms_per_step": d.get("ms_per_step"), "steps": d.get("steps"), "warmup": d.get("warmup"),
                "wall_s": round(time.time() - t0, 1), "argv": " ".join(argv)}
        rf = d.get("roofline")
        if rf:
            summ["roofline"] = {k: rf.get(k) for k in ("bound", "achieved", "peak", "unit", "frac", "kernel")}
        cfg = d.get("config", {})
        for k in ("partitioned_pass_ms", "launch_shape", "rows", "commands", "launches_per_run"):
            if k in cfg:
                summ[k] = cfg[k]
        for k in ("plain", "clocks", "cpu_baseline", "parity"):
            if k in d:
                summ[k] = d[k]
        rg = d.get("reference_gpu")
        if rg:
            summ["reference_gpu"] = {k: rg.get(k) for k in ("value", "ms_per_pass", "kernel_ms_per_pass",
                                                           "parity", "unavailable", "error") if k in rg}
        out[name] = summ
    return out


def run_reference(args, rank, world):
    if rank != 0:
        return
    t0 = time.time()
    nrows = min(args.rows, 20_000_000)
    fact, sess, km, chunks, meta = build_workload(nrows, 0)
    threads = os.cpu_count() or 1
    per_step = max(2.0, min(args.cpu_seconds, 120.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_rows_per_sec(sess, km, chunks, per_step / 2, threads)
    vals, total_rows, total_s, kind = [], 0, 0.0, "port"
    for _ in range(args.steps):
        v, kind, rows, el = cpu_rows_per_sec(sess, km, chunks, per_step, threads)
        vals.append(v)
        total_rows += rows
        total_s += el
    value = total_rows / total_s
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
            "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * total_s / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic",
            "config": {"workload": "two-way hash join + group-by, heap, 100M-row fact "
                                   "(bounded sample per step, see cpu_baseline)",
                       "fact_rows_generated": nrows, "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"{total_rows} fact rows over {total_s:.1f} s "
                                       f"({per_step:.1f} s per step) of the same workload"},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------ GPU arm
def run_b200(args, rank, world, local):
    import torch
    import xb_final as F
    import xpu_b200
    torch.cuda.set_device(local)
    fact, sess, km, chunks, meta = build_workload(args.rows, rank)
    nbytes = sum(c.nbytes for c in chunks)
    dev = xpu_b200.Device(local)

    # ---- value: chunks resident in HBM, one persistent launch per step
    s = xpu_b200.Session(dev, sess, km, 2)
    ups = [dev.upload(c) for c in chunks]
    batch = s.batch([p for _, p in ups])
    shape = _tune(batch, args)
    r = batch.exec()
    assert r["nitems_raw"] == meta["nitems_raw"], r
    for _ in range(max(0, args.warmup - 1)):
        batch.exec()
    sampler = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    sampler.start()
    ms = batch.time(args.steps)                 # CUDA events around each launch
    torch.cuda.synchronize()
    barrier(world)
    clocks = sampler.stop()
    ms_max = max_over_ranks(ms, world)
    rows_total = sum_over_ranks(float(args.rows), world)
    value = rows_total / (ms_max / 1000.0)
    # sanity: the batch really did the work
    r2 = batch.exec()
    assert r2["nitems_out"] == meta["nitems_out"], (r2, meta)
    info = s.info()
    kernel = ("xbj_kernel (session-specialised, NVRTC sm_100a)" if "jit" in info["kernels"].values()
              else "xb_exec_kernel (interpreter)")
    batch.close()
    s.close()
    # parity at full size: one pass of the timed batch path on a fresh
    # session, its kds_final decoded and compared with the generator's
    # per-region truth (int128 sums and counts, exact)
    sp = xpu_b200.Session(dev, sess, km, 2)
    bp = sp.batch([p for _, p in ups])
    bp.exec()
    bp.close()
    final_b, _ = sp.final()
    sp.close()
    batch_errs = F.compare_groups(F.decode_kds_final(final_b, sess), meta["truth"], rtol=0.0)
    assert batch_errs == [], batch_errs[:3]

    # ---- e2e: whole query through the C ABI from pinned host memory
    pinned = []
    for c in chunks:
        t = torch.empty(c.nbytes, dtype=torch.uint8, pin_memory=True)
        t.numpy()[:] = c
        pinned.append(t)
    km_pinned = torch.empty(km.nbytes, dtype=torch.uint8, pin_memory=True)
    km_pinned.numpy()[:] = km
    kmp = km_pinned.numpy()
    e2e_times, d2h = [], 0
    for it in range(args.e2e_steps + 1):
        barrier(world)
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        se = xpu_b200.Session(dev, sess, kmp, 2)
        for t in pinned:
            se.exec(t.numpy())
        final, res = se.final()
        se.close()
        torch.cuda.synchronize()
        el = time.perf_counter() - t0
        barrier(world)
        d2h = final.nbytes if final is not None else 0
        if it > 0:                                 # first pass is warm-up
            e2e_times.append(el)
    e2e_el = max_over_ranks(sum(e2e_times) / len(e2e_times), world)
    e2e_value = rows_total / e2e_el
    e2e_errs = F.compare_groups(F.decode_kds_final(final, sess), meta["truth"], rtol=0.0)
    assert e2e_errs == [], e2e_errs[:3]
    parity = {"groups": len(meta["truth"]), "rows_checked_per_gpu": args.rows,
              "batch_equals_truth": True, "e2e_equals_truth": True,
              "compared": "every group's int128 sum(qty*price) and count(*), exact, against the "
                          "generator's column arrays"}

    # ---- N>1: every rank's kds_final merged on rank 0's GPU (the service's
    # final step over per-GPU results); checked against the ranks' row counts
    merge = None
    if world > 1 and args.final_merge == "exchange":
        import xb_exchange as X
        # a session holding this rank's groups, split and exchanged on the
        # devices (not part of the timed value)
        sx = xpu_b200.Session(dev, sess, kmp, 2)
        for t in pinned:
            sx.exec(t.numpy())
        t0 = time.perf_counter()
        share = X.exchange_final(dev, sess, sx, rank, world, kmp, 2, device=f"cuda:{local}")
        sx.close()
        ms_x = max_over_ranks(1000.0 * (time.perf_counter() - t0), world)
        mine = F.decode_kds_final(share, sess) if share is not None else {}
        groups = sum_over_ranks(float(len(mine)), world)
        rows = sum_over_ranks(float(sum(v[1] for v in mine.values())), world)
        nout = sum_over_ranks(float(meta["nitems_out"]), world)
        assert rows == nout, "exchanged row count"
        merge = {"ranks": world, "groups": int(groups), "ms": ms_x,
                 "includes": "FinalParts (split by hash % N on each GPU), NCCL all-to-all of the parts "
                             "between the GPUs' memories, MergeFinal of the received parts from device "
                             "memory into a fresh session, Final"}
    elif world > 1:
        finals = gather_finals(final, rank, world)
        nout = sum_over_ranks(float(meta["nitems_out"]), world)
        if rank == 0:
            t0 = time.perf_counter()
            sm = xpu_b200.Session(dev, sess, kmp, 2)
            for f in finals:
                if f is not None:
                    sm.merge_final(f)
            merged, _ = sm.final()
            sm.close()
            merge_ms = 1000.0 * (time.perf_counter() - t0)
            groups = F.decode_kds_final(merged, sess)
            assert sum(v[1] for v in groups.values()) == int(nout), "merged row count"
            merge = {"ranks": world, "groups": len(groups), "ms": merge_ms,
                     "includes": "OpenSession, one MergeFinal per rank's kds_final (host copy), Final"}
        barrier(world)

    # ---- CPU baseline (rank 0, N=1 only)
    cpu = None
    if rank == 0 and world == 1:
        threads = os.cpu_count() or 1
        v, kind, rows, el = cpu_rows_per_sec(sess, km, chunks[:8], args.cpu_seconds, threads)
        cpu = {"value": v, "unit": UNIT, "cores": threads, "kind": kind,
               "sample": f"{rows} fact rows of the same workload in {el:.1f} s on {threads} threads "
                         f"({'PG-Strom expression library host-compiled from the reference' if kind == 'reference' else 'C restatement'})"}

    # ---- served mix (rank 0, N=1): continuous batching against the plain drop-in
    served = None
    if rank == 0 and world == 1 and args.served_leg:
        try:
            served = served_leg(dev)
        except Exception as e:          # the headline stands without it
            served = {"error": f"{type(e).__name__}: {e}"[:300]}

    # ---- the other configurations (rank 0, N=1), each in its own process
    configs = None
    if rank == 0 and world == 1 and args.configs:
        configs = config_lines()

    # ---- the reference's own kernel on this GPU (rank 0, N=1), after
    # every other measurement of the line
    ref_gpu_line = None
    if rank == 0 and world == 1 and args.reference_gpu:
        try:
            ref_gpu_line = reference_gpu_leg(sess, km, chunks, args.rows, meta["truth"], rtol=0.0)
        except Exception as e:          # the headline stands without it
            ref_gpu_line = {"error": f"{type(e).__name__}: {e}"[:300]}

    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = nbytes / (ms / 1000.0) / 1e9
    traffic = None
    prof = os.path.join(ROOT, "profiles", "traffic_join_groupby.json")
    if os.path.exists(prof):
        try:
            traffic = json.load(open(prof))["bytes_per_algorithmic_byte"] * nbytes
        except (OSError, KeyError, ValueError):
            traffic = None
    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max,
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
                "dtype": "int64", "data": "synthetic (seeded; shapes/distributions of the config)",
                "config": {"workload": "two-way hash join + group-by over heap pages: "
                                       f"{args.rows // 1_000_000}M-row fact x dim1 200k x dim2 10k, "
                                       "GROUP BY region -> sum(qty*price), count(*)",
                           "fact_rows_per_gpu": args.rows, "chunks_per_gpu": len(chunks),
                           "chunk_bytes": "64 MB KDS_FORMAT_BLOCK", "heap_bytes_per_gpu": nbytes,
                           "l2_note": "inputs (5.2 GB) exceed L2 (126 MB) by 40x",
                           "parallelism": f"dp{world} (independent shards, no collective)",
                           "launch_shape": shape},
                "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                             "frac": achieved / peak, "traffic": traffic,
                             "kernel": kernel,
                             "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback"},
                "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": nbytes + km.nbytes + len(sess),
                        "d2h_bytes_per_step": d2h, "ms_per_step": 1000.0 * e2e_el,
                        "includes": "OpenSession (dims upload + device index build), ExecTask per 64 MB "
                                    "chunk from pinned host memory, Final read-back, CloseSession"},
                "clocks": clocks,
                "gpu_launches": args.steps,
                "parity": parity,
                "cpu_baseline": cpu}
        if served:
            line["served"] = served
        if ref_gpu_line:
            line["reference_gpu"] = ref_gpu_line
        if configs:
            line["configs"] = configs
        if merge:
            line["final_merge"] = merge
        print(json.dumps(line), flush=True)
    for base, _ in ups:
        dev.free(base)
    dev.close()


# ------------------------------------------------------------------ other configurations
# The reference's functions keep one session's groups per host thread: the
# CPU arms read the Arrow configuration in chunks of this many rows, so that
# a thread holds tens of thousands of groups rather than the half million of
# a 2.5M-row chunk (about 50 MB against 460 MB per thread)
CPU_ARROW_CHUNK_ROWS = 250_000


def _config_workload(args, nrows, rows_per_chunk=None):
    """(chunks, session, truth or None, meta, description, referenced bytes)
    of the scan or Arrow configuration at nrows (rows_per_chunk: Arrow
    chunks of that many rows instead of the configuration's)"""
    import xb_configs as C
    if args.workload == "scan_groupby":
        tbl, sess, _, expect, meta = C.scan_groupby(nrows=nrows)
        chunks = tbl.block_chunks(pages_per_chunk=8190)
        desc = (f"plain scan + filter + group-by over heap pages: {nrows} rows, WHERE a < 300 "
                "GROUP BY g (64 groups) -> count, sum(a), sum(c numeric), avg(b)")
        truth = {k: [v["nrows"], v["sum_a"], v["sum_c"], v["avg_b"]] for k, v in expect.items()}
        return chunks, sess, truth, meta, desc, sum(c.nbytes for c in chunks)
    kw = {"rows_per_chunk": rows_per_chunk} if rows_per_chunk else {}
    chunks, sess, _, meta = C.arrow_groupby(nrows=nrows, nkeys=args.keys, with_expect=False, **kw)
    desc = (f"Arrow high-cardinality pre-aggregation: {nrows} rows, {args.keys} keys, 2-year date "
            "window -> GROUP BY k: count, sum(v1), min/max/sum(v2)")
    return chunks, sess, None, meta, desc, 24 * nrows


def run_reference_config(args):
    """The reference arm of the scan and Arrow configurations: the
    reference's host-compiled functions on every host thread, over a
    bounded sample of the same workload per step."""
    nrows = min(args.rows, 20_000_000)
    arrow = args.workload != "scan_groupby"
    chunks, sess, _, meta, desc, _ = _config_workload(args, nrows,
                                                      CPU_ARROW_CHUNK_ROWS if arrow else None)
    threads = os.cpu_count() or 1
    per_step = max(2.0, min(args.cpu_seconds, 120.0 / max(1, args.steps + args.warmup)))
    for _ in range(args.warmup):
        cpu_rows_per_sec(sess, None, chunks, per_step / 2, threads)
    total_rows, total_s, kind = 0, 0.0, "port"
    for _ in range(args.steps):
        v, kind, rows, el = cpu_rows_per_sec(sess, None, chunks, per_step, threads)
        total_rows += rows
        total_s += el
    value = total_rows / total_s
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * total_s / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic", "config": {"workload": desc + " (bounded sample per step)",
                                            "rows_generated": nrows, "parallelism": "host threads"},
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": kind,
                             "sample": f"{total_rows} rows over {total_s:.1f} s ({per_step:.1f} s per step)"
                                       + (f", in {CPU_ARROW_CHUNK_ROWS}-row chunks" if arrow else "")},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def run_config(args):
    """One persistent launch per pass over resident chunks of the plain
    scan + group-by table (heap) or the Arrow high-cardinality table;
    rows/s and the referenced bytes against HBM bandwidth."""
    import torch
    import xpu_b200
    t0 = time.time()
    # heap: every chunk byte; Arrow: k, v1, v2, d, the referenced columns
    chunks, sess, truth, meta, desc, ref_bytes = _config_workload(args, args.rows)
    nbytes = sum(c.nbytes for c in chunks)
    gen_s = time.time() - t0
    dev = xpu_b200.Device(0)
    s = xpu_b200.Session(dev, sess)
    ups = [dev.upload(c) for c in chunks]
    batch = s.batch([p for _, p in ups])
    shape = _tune(batch, args)
    r = batch.exec()
    assert r["nitems_raw"] == meta["nitems_raw"], r
    if truth is not None:
        import xb_final as F
        final, _ = s.final()
        assert F.compare_groups(F.decode_kds_final(final, sess), truth) == []
    for _ in range(max(0, args.warmup - 1)):
        batch.exec()
    sampler = ClockSampler(0)
    torch.cuda.synchronize()
    sampler.start()
    ms = batch.time(args.steps)
    clocks = sampler.stop()
    info = s.info()
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = ref_bytes / (ms / 1000.0) / 1e9
    line = {"metric": METRIC, "value": args.rows / (ms / 1000.0), "unit": UNIT, "n_gpus": 1,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "int64", "data": "synthetic (seeded)",
            "config": {"workload": desc, "rows": args.rows, "chunks": len(chunks), "chunk_bytes": nbytes,
                       "generation_s": round(gen_s, 1), "launch_shape": shape,
                       **({"partitioned_pass_ms": {"scan": round(info["last_part_scan_ms"], 3),
                                                   "replay": round(info["last_part_replay_ms"], 3)}}
                          if info.get("partition_used") else {})},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None, "algorithmic_bytes": ref_bytes,
                         "kernel": ("xbj_kernel" if "jit" in info["kernels"].values() else "xb_exec_kernel"),
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback"},
            "clocks": clocks, "gpu_launches": args.steps,
            "parity": ({"groups_equal_truth": True,
                        "compared": "every group of the first pass against the generator's column arrays: "
                                    "counts, integer and numeric sums exact; float8 averages within 1e-12 "
                                    "relative (of the sum of magnitudes where a group's terms cancel)"}
                       if truth is not None else
                       {"checked": False,
                        "why": "no truth is generated at this size; the GPU tests check the same session "
                               "shape against the truth up to 2M rows / 1M keys"})}
    if args.workload == "scan_groupby" and args.reference_gpu:
        try:
            line["reference_gpu"] = reference_gpu_leg(sess, None, chunks, args.rows, truth)
        except Exception as e:
            line["reference_gpu"] = {"error": f"{type(e).__name__}: {e}"[:300]}
    if args.cpu_seconds > 0:
        threads = os.cpu_count() or 1
        cchunks = chunks[:8]
        if args.workload != "scan_groupby":
            cchunks = _config_workload(args, 8 * CPU_ARROW_CHUNK_ROWS, CPU_ARROW_CHUNK_ROWS)[0]
        v, kind, rows, el = cpu_rows_per_sec(sess, None, cchunks, args.cpu_seconds, threads)
        line["cpu_baseline"] = {"value": v, "unit": UNIT, "cores": threads, "kind": kind,
                                "sample": f"{rows} rows of the same workload in {el:.1f} s on {threads} threads "
                                          + (f"in {CPU_ARROW_CHUNK_ROWS}-row chunks "
                                             if args.workload != "scan_groupby" else "")
                                          + f"({'PG-Strom expression library host-compiled from the reference' if kind == 'reference' else 'C restatement'})"}
    print(json.dumps(line), flush=True)
    batch.close()
    s.close()
    for b, _ in ups:
        dev.free(b)
    dev.close()


# ------------------------------------------------------------------ batched commands
def run_mixed(args):
    """256 chunk commands on the plain scan schema (one session each; chunk
    sizes log-uniform 64 KB-64 MB, selectivity U[0.1%,90%], group counts
    log-uniform 1-1M) as one mixed batch: one persistent launch per kernel,
    replayed from a captured CUDA graph.  Beside it: the same commands as
    plain per-command xpuB200ExecTask calls on the same resident chunks."""
    import torch
    import xb_configs as C
    import xpu_b200
    t0 = time.time()
    cmds = C.mixed_commands(ncmds=256)
    gen_s = time.time() - t0
    dev = xpu_b200.Device(0)
    ups = [dev.upload(c["chunk"]) for c in cmds]
    # launch shape tuned on the largest command (a session of its own); the
    # commands' sessions adopt its CTA bound at their first launch
    shape = {"tuned": False}
    if args.tune:
        big = max(range(len(cmds)), key=lambda i: cmds[i]["chunk"].nbytes)
        ts = xpu_b200.Session(dev, cmds[big]["session"])
        tb = ts.batch([ups[big][1]])
        shape = _tune(tb, args)
        shape["tuned_on"] = f"command {big} ({cmds[big]['chunk'].nbytes} bytes)"
        tb.close()
        ts.close()
    sessions = [xpu_b200.Session(dev, c["session"]) for c in cmds]
    mix = xpu_b200.Mix(dev, sessions, [p for _, p in ups])
    out = mix.exec()
    assert all(err is None for _, err in out), [str(e) for _, e in out if e][:3]
    for (r, _), c in zip(out, cmds):
        assert r["nitems_in"] == c["meta"]["nitems_in"]
    for _ in range(max(0, args.warmup - 1)):
        mix.exec()
    sampler = ClockSampler(0)
    torch.cuda.synchronize()
    sampler.start()
    ms = mix.time(args.steps)
    clocks = sampler.stop()
    info = mix.info()
    rows = sum(c["params"]["rows"] for c in cmds)
    # plain drop-in: one ExecTask per command, each waiting for its result
    for s, (_, p) in zip(sessions, ups):
        s.exec(p, on_device=True)
    torch.cuda.synchronize()
    t1 = time.perf_counter()
    for _ in range(args.steps):
        for s, (_, p) in zip(sessions, ups):
            s.exec(p, on_device=True)
    plain_ms = 1000.0 * (time.perf_counter() - t1) / args.steps
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except OSError:
        pass
    peak = peaks.get("hbm_gbs", 6650.0)
    achieved = info["bytes"] / (ms / 1000.0) / 1e9
    line = {"metric": "batched chunk commands rows/s", "value": rows / (ms / 1000.0), "unit": "rows/s",
            "n_gpus": 1, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "int64",
            "data": "synthetic (seeded)",
            "config": {"workload": "256 scan/pre-agg commands on the plain scan schema, chunks log-uniform "
                                   "64 KB-64 MB, selectivity U[0.1%,90%], group counts log-uniform 1-1M",
                       "commands": len(cmds), "rows": rows, "chunk_bytes": info["bytes"],
                       "launches_per_run": info["launches"], "specialised_commands": info["specialised"],
                       "work_items": info["items"], "generation_s": round(gen_s, 1),
                       "launch_shape": shape,
                       "l2_note": "inputs (2.2 GB) exceed L2 (126 MB)"},
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": None,
                         "peak_source": "MEASURED_PEAKS.json hbm_gbs (of measured)" if peaks else "fallback"},
            "plain": {"ms_per_run": plain_ms, "rows_per_s": rows / (plain_ms / 1000.0),
                      "how": "one xpuB200ExecTask per command on the same resident chunks, sequential"},
            "parity": {"rows_in_equal_truth": True,
                       "compared": "every command's qualifying-row count against its generator; the groups "
                                   "of a mixed batch against the truth and the oracle: tests/test_gpu_mixed.py"},
            "clocks": clocks, "gpu_launches": args.steps * info["launches"]}
    print(json.dumps(line), flush=True)
    mix.close()
    for s in sessions:
        s.close()
    for b, _ in ups:
        dev.free(b)
    dev.close()


# ------------------------------------------------------------------ served mix
class _Tables:
    """The three query templates' tables, resident in HBM through the
    library's chunk cache (xpuB200ChunkCachePut), as a service keeps its
    cached tables across requests."""

    def __init__(self, dev, rows0, rows1, rows2):
        import xb_configs as C
        self.bytes = 0
        self.handle = 0x7AB0

        def up(chunks):
            self.bytes += sum(c.nbytes for c in chunks)
            self.handle += 1
            return [(None, dev.chunk_put(self.handle, i, c)) for i, c in enumerate(chunks)]
        tbl0, _, _, _, _ = C.scan_groupby(nrows=rows0, seed_config=20)
        self.t0 = up(tbl0.block_chunks(pages_per_chunk=8190))
        self.rows0 = rows0
        del tbl0
        fact, _, km, _, _ = C.join_groupby(nfact=rows1, seed_config=21)
        self.t1 = up(fact.block_chunks(pages_per_chunk=8190))
        self.km = km
        self.rows1 = rows1
        del fact
        chunks2, _, _, _ = C.arrow_groupby(nrows=rows2, nkeys=10_000_000, seed_config=22,
                                           rows_per_chunk=2_500_000, with_expect=False)
        self.t2 = up(chunks2)
        self.rows2 = rows2

    def free(self, dev):
        for t in (self.t0, self.t1, self.t2):
            for _, p in t:
                dev.chunk_release(p)
        dev.chunk_cache(0)                  # the released chunks leave
        dev.chunk_cache(64 << 30)           # the default budget again


INNER_HANDLE_DIMS = 0xD1D2      # join_inner_handle of the join template's dimension tables


def _requests(tables, n, qps, seed=0x5EED):
    """Poisson arrivals; templates 50/30/20; rows log-uniform from 1M to
    the table; randomized predicate constants."""
    import xb_configs as C
    r = np.random.default_rng(seed)
    t, out = 0.0, []
    for i in range(n):
        t += r.exponential(1.0 / qps)
        u = r.random()
        if u < 0.5:
            rows = int(np.exp(r.uniform(np.log(1e6), np.log(tables.rows0))))
            k = max(1, round(rows / tables.rows0 * len(tables.t0)))
            sess = C.scan_groupby_session(a_limit=int(r.integers(1, 1000)), ngroups=64)
            out.append({"t": t, "tpl": 0, "session": sess, "km": None, "nrels": 0,
                        "chunks": [p for _, p in tables.t0[:k]]})
        elif u < 0.8:
            rows = int(np.exp(r.uniform(np.log(1e6), np.log(tables.rows1))))
            k = max(1, round(rows / tables.rows1 * len(tables.t1)))
            fl = int(r.integers(1, 5))
            sess = C.join_groupby_session(flag_limit=fl)
            # the serving path names the (unchanging) dimension tables, so
            # their device indexes stay resident across requests
            served_sess = C.join_groupby_session(flag_limit=fl, inner_handle=INNER_HANDLE_DIMS)
            out.append({"t": t, "tpl": 1, "session": sess, "session_served": served_sess,
                        "km": tables.km, "nrels": 2, "chunks": [p for _, p in tables.t1[:k]]})
        else:
            rows = int(np.exp(r.uniform(np.log(1e6), np.log(tables.rows2))))
            k = max(1, round(rows / tables.rows2 * len(tables.t2)))
            lo = 16436 + int(r.integers(0, 3652 - 730))
            est = min(10_000_000, k * 2_500_000 // 5)
            sess = C.arrow_groupby_session(lo_day=lo, hi_day=lo + 730, ngroups_estimate=est)
            out.append({"t": t, "tpl": 2, "session": sess, "km": None, "nrels": 0,
                        "chunks": [p for _, p in tables.t2[:k]]})
    return out


def _serve_plain(dev, reqs, start):
    """One query at a time in arrival order: OpenSession, ExecTask per
    chunk, Final, CloseSession (the plain drop-in)."""
    import xpu_b200
    lat = []
    for q in reqs:
        while time.perf_counter() - start < q["t"]:
            pass
        s = xpu_b200.Session(dev, q["session"], q["km"], q["nrels"])
        for p in q["chunks"]:
            s.exec(p, on_device=True)
        s.final()
        s.close()
        lat.append(time.perf_counter() - start - q["t"])
    return lat, time.perf_counter() - start


MAX_ACTIVE = 16                 # queries admitted at once (each holds its group table)
FINAL_THREADS = 4               # kds_final read-backs in flight
FINAL_BUF_BYTES = 1536 << 20    # pinned response buffer per read-back


def _pinned_buffers(nbytes=FINAL_BUF_BYTES):
    import queue
    import torch
    q = queue.Queue()
    for _ in range(FINAL_THREADS):
        q.put(torch.empty(nbytes, dtype=torch.uint8, pin_memory=True).numpy())
    return q


def _served_compare(dev, tables, requests, qps, bufs):
    """The served and plain forms over the same requests: open-loop p50 /
    p99 at the offered rate and saturation throughput (every query queued
    at once), after a warm-up of both."""
    reqs = _requests(tables, requests, qps)
    warm = _requests(tables, 30, qps, seed=7)
    served = lambda d, r, t: _serve_batched(d, r, t, bufs)
    _serve_plain(dev, warm, time.perf_counter())      # kernel cache, pools
    served(dev, warm, time.perf_counter())
    res = {}
    for mode, fn in (("plain", _serve_plain), ("served", served)):
        lat, el = fn(dev, reqs, time.perf_counter())
        sat = [dict(q, t=0.0) for q in reqs]
        _, sat_el = fn(dev, sat, time.perf_counter())
        res[mode] = {"qps": len(reqs) / el, "p50_ms": 1000 * float(np.percentile(lat, 50)),
                     "p99_ms": 1000 * float(np.percentile(lat, 99)),
                     "saturation_qps": len(reqs) / sat_el}
    mix = {k: sum(1 for q in reqs if q["tpl"] == k) for k in range(3)}
    return res, mix


def served_leg(dev, requests=100, qps=200.0):
    """A short served-mix measurement for the headline line: 100 Poisson
    requests (mean 200 QPS) over resident tables of 8M (scan), 20M (join)
    and 20M (Arrow) rows, served and plain."""
    t0 = time.time()
    tables = _Tables(dev, rows0=8_000_000, rows1=20_000_000, rows2=20_000_000)
    gen_s = time.time() - t0
    try:
        res, mix = _served_compare(dev, tables, requests, qps, _pinned_buffers(512 << 20))
    finally:
        tables.free(dev)
    return {"requests": requests, "offered_qps": qps, "template_counts": mix,
            "tables_rows": [8_000_000, 20_000_000, 20_000_000], "generation_s": round(gen_s, 1),
            "qps": res["served"]["qps"], "p50_ms": res["served"]["p50_ms"],
            "p99_ms": res["served"]["p99_ms"], "saturation_qps": res["served"]["saturation_qps"],
            "plain_qps": res["plain"]["qps"], "plain_p50_ms": res["plain"]["p50_ms"],
            "plain_p99_ms": res["plain"]["p99_ms"], "plain_saturation_qps": res["plain"]["saturation_qps"],
            "saturation_ratio": res["served"]["saturation_qps"] / res["plain"]["saturation_qps"]}


def _serve_batched(dev, reqs, start, bufs):
    """Continuous batching: a query's chunks are submitted when it arrives
    and a query slot is free; finished queries are finalised (kds_final read
    back) by worker threads while other queries run on the GPU."""
    from concurrent.futures import ThreadPoolExecutor
    import xpu_b200
    lat = [None] * len(reqs)
    running, finishing = {}, {}
    nxt, ndone = 0, 0

    def finish(i, s):
        buf = bufs.get()
        try:
            s.final(out=buf)
        finally:
            bufs.put(buf)
        s.close()
        lat[i] = time.perf_counter() - start - reqs[i]["t"]

    with ThreadPoolExecutor(max_workers=FINAL_THREADS) as pool:
        while ndone < len(reqs):
            now = time.perf_counter() - start
            while (nxt < len(reqs) and reqs[nxt]["t"] <= now and
                   len(running) + len(finishing) < MAX_ACTIVE):
                q = reqs[nxt]
                s = xpu_b200.Session(dev, q.get("session_served", q["session"]), q["km"], q["nrels"])
                running[nxt] = (s, [dev.submit(s, p, on_device=True) for p in q["chunks"]])
                nxt += 1
            for i in list(running):
                s, tickets = running[i]
                left = [t for t in tickets if dev.poll(t, nrels=reqs[i]["nrels"], wait=False) is None]
                if left:
                    running[i] = (s, left)
                    continue
                del running[i]
                finishing[i] = pool.submit(finish, i, s)
            for i in list(finishing):
                if finishing[i].done():
                    finishing.pop(i).result()
                    ndone += 1
    return lat, time.perf_counter() - start


def run_served(args):
    """Served mixed workload: Poisson arrivals (mean --qps) of queries drawn
    50/30/20 from the three templates over device-resident tables, served
    by the plain drop-in (one query at a time) and by the serving scheduler
    (Submit/Poll, continuous batching).  Open-loop latency p50/p99 at the
    offered rate, and saturation throughput (every query queued at once)."""
    import xpu_b200
    dev = xpu_b200.Device(0)
    t0 = time.time()
    tables = _Tables(dev, rows0=16_000_000, rows1=50_000_000, rows2=args.served_arrow_rows)
    gen_s = time.time() - t0
    res, mix = _served_compare(dev, tables, args.requests, args.qps, _pinned_buffers())
    line = {"metric": "served QPS (p50/p99 latency)", "value": res["served"]["saturation_qps"],
            "unit": "queries/s", "n_gpus": 1, "higher_is_better": True, "vs_baseline": None,
            "dtype": "int64", "data": "synthetic (seeded)",
            "config": {"workload": "Poisson arrivals, templates 50/30/20 (scan+group-by 16M-row heap, "
                                   "two-way join 50M-row heap, Arrow group-by "
                                   f"{args.served_arrow_rows // 1_000_000}M rows), rows log-uniform "
                                   "1M..table per query, randomized constants, tables resident in HBM",
                       "requests": args.requests, "offered_qps": args.qps, "template_counts": mix,
                       "resident_bytes": tables.bytes, "generation_s": round(gen_s, 1)},
            "served": res["served"], "plain": res["plain"],
            "served_inner_cache_bytes": dev.inner_cache(),
            "saturation_ratio": res["served"]["saturation_qps"] / res["plain"]["saturation_qps"]}
    print(json.dumps(line), flush=True)
    tables.free(dev)
    dev.close()


def main():
    args = parse()
    if args.workload != "join_groupby":
        if args.impl == "reference":
            if args.workload in ("scan_groupby", "arrow_groupby"):
                return run_reference_config(args)
            print(json.dumps({"impl": "reference", "unavailable": "the reference has no batched or served "
                                                                  "form of this path"}), flush=True)
            return
        if args.workload in ("scan_groupby", "arrow_groupby"):
            return run_config(args)
        return run_mixed(args) if args.workload == "mixed" else run_served(args)
    rank, world, local = dist_setup(args.gpus)
    try:
        if args.impl == "reference":
            run_reference(args, rank, world)
        else:
            run_b200(args, rank, world, local)
    finally:
        if world > 1:
            import torch.distributed as dist
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the LSD radix-sort hot path on B200.

Workload (one "step"): a stable ascending LSD sort of 2^28 (268,435,456) uint32 keys drawn
uniform over [0, 2^32) from seeded PCG32 streams -- the plain-sort-at-scale configuration
the headline metric is quoted on.  Other dtypes/configs are parity-test cases.

Arms
  default (ours)   value: device-resident sorts through the C ABI (*_dev), CUDA events
                   around each step on the context's stream, K steps over distinct copies
                   of the input (inputs 1 GiB each > L2, restored between steps outside the
                   events); e2e: the host-array C ABI call (H2D, sort, D2H into the same
                   array) timed around each synchronous call, on a pageable host array (what a
                   fixed .NET array is; e2e) and on a pinned one (e2e_pinned).
  --impl reference the CPU restatement of the reference's SortRadixPar (oracle, all host
                   threads) on a bounded sample of the same keys per step.

Multi-GPU (torchrun): the plain sort does not shard (each digit pass is a global
permutation), so N ranks run N independent replicas ("replicas only", weak scaling);
value = keys sorted by all ranks / max-over-ranks time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "Gkeys/s & % HBM roofline (256M u32); batched/served vs plain, p50/p99, 1 B200"
UNIT = "Gkeys/s"
N_DEFAULT = 1 << 28
FALLBACK_HBM_GBS = 6650.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--n", type=int, default=N_DEFAULT)
    ap.add_argument("--dtype", default="u32", choices=["u32", "i32", "f32", "u64", "i64", "f64"])
    ap.add_argument("--scheme", default="auto", choices=["auto", "chunked", "lookback"],
                    help="plain: the digit-pass scheme of the library (auto picks by key type and n)")
    ap.add_argument("--slots", type=int, default=4, help="distinct input copies cycled through")
    ap.add_argument("--e2e-steps", type=int, default=0, help="0 = same as --steps (capped at 20)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--workload", default="plain",
                    choices=["plain", "batched", "served", "configs", "sharded", "kernels"],
                    help="plain: the 2^28-key sort (headline); batched: 65,536 mixed arrays; "
                         "served: Poisson sort/top-k requests swept to saturation; configs: every "
                         "plain-sort and pairs configuration, device-resident; sharded: one array of "
                         "--n keys per rank sorted across the ranks (partition, NCCL all-to-all, "
                         "local sort, rebalance); kernels: radix top-k, in-place SelectTopK and "
                         "the 8/16-bit counting sorts, device-resident")
    ap.add_argument("--requests", type=int, default=120, help="served: requests per arrival rate")
    ap.add_argument("--loads", default="0.25,0.5,1,2,4,8,16",
                    help="served: offered loads, as multiples of the plain form's capacity")
    ap.add_argument("--arrays", type=int, default=65536,
                    help="batched: number of arrays (the scaled total keeps ~3,815 keys per array)")
    ap.add_argument("--literal", action="store_true",
                    help="batched: the literal length distribution (~6.6 G keys) instead of ~250 M")
    return ap.parse_args()


# ---------------------------------------------------------------------------------------
def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index: int):
        self.idx = device_index
        self.proc = None
        self.lines = []
        self._t = None

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.idx}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "100"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        if self._t:
            self._t.join(timeout=2)
        sm, smax, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": smax,
                "reasons": sorted(reasons), "samples": len(sm)}


def _in_order(a: np.ndarray) -> bool:
    """Ascending in the library's key order (signed by value; floats by the sign-flip order)."""
    u = a.view(np.uint32 if a.dtype.itemsize == 4 else np.uint64)
    top = u.dtype.type(1) << u.dtype.type(8 * a.dtype.itemsize - 1)
    if a.dtype.kind == "i":
        u = u ^ top
    elif a.dtype.kind == "f":
        u = np.where((u & top) != 0, ~u, u ^ top)
    return bool(np.all(u[1:] >= u[:-1]))


def gen_keys(dtype: str, n: int, seed: int = 1) -> np.ndarray:
    from hpcsharp_b200 import datagen

    return datagen.by_name(dtype, n, seed)


def read_traffic(dtype: str):
    """DRAM bytes per digit-pass launch from the committed ncu summary, if present."""
    p = os.path.join(ROOT, "profiles", f"chunk_pass_{dtype}_256M.txt")
    try:
        for line in open(p):
            if line.startswith("dram_bytes_per_launch="):
                return float(line.split("=", 1)[1])
    except OSError:
        pass
    return None


# ---------------------------------------------------------------------------------------
def cpu_baseline(dtype: str, n: int, budget_s: float = 15.0):
    """The oracle's SortRadixPar restatement on all host cores, scratch allocated once outside the
    timed calls.  u32 (the headline): the full n-key configuration, best of 3.  Other key types:
    the largest power-of-two sample whose 3 repetitions fit the budget."""
    import oracle

    oracle.build()
    th = oracle.hardware_threads()
    if dtype == "u32":
        sample = n
        a = oracle.gen_u32_uniform(n, seed=1, threads=th)
    else:
        sample = min(n, 1 << 24)
        a = gen_keys(dtype, sample, seed=7)
    ws = oracle.RadixParWorkspace(n, a.dtype.itemsize)
    b = np.empty_like(a)

    def once():
        np.copyto(b, a)
        t0 = time.perf_counter()
        ws.sort(b, threads=th)
        return time.perf_counter() - t0

    dt = once()
    # grow the sample while the projected time for 3 repetitions stays inside the budget
    while dtype != "u32" and sample * 2 <= n and dt * 2 * 3 < budget_s:
        sample *= 2
        a = gen_keys(dtype, sample, seed=7)
        b = np.empty_like(a)
        dt = once()
    best = min(once() for _ in range(3))
    ws.close()
    what = "the full configuration" if sample == n else f"a {sample}-key sample of the same generator"
    return {"value": round(sample / best / 1e9, 4), "unit": UNIT, "cores": th, "kind": "port",
            "sample": f"{what} ({sample} {dtype} keys), SortRadixPar C++ restatement (fully parallel, 64 Ki "
                      f"quanta), scratch allocated once outside the timed calls, best of 3"}


def plain_config(n: int, dtype: str, world: int, digest: str) -> dict:
    """The plain-sort workload's config, the same dict in both arms (ours and the reference)."""
    w = 4 if dtype in ("u32", "i32", "f32") else 8
    return {"workload": f"plain LSD radix sort of {n} {dtype} keys uniform over the key range, stable, "
                        f"8-bit digits",
            "n": n, "parallelism": f"replicas x{world}", "input_sha256": digest,
            "l2": f"inputs {'larger' if n * w > 126 * 2**20 else 'smaller'} than L2 ({n * w} bytes per copy)"}


def input_digest(a: np.ndarray) -> str:
    """SHA-256 of the keys a step sorts: both arms print it, so their inputs can be compared."""
    import hashlib

    return hashlib.sha256(memoryview(a).cast("B")).hexdigest()


def run_reference(args, rank: int, world: int):
    """--impl reference: the reference's SortRadixPar (C++ restatement of RadixSortLsdParallel.cs:
    145-232; the C# reference needs .NET, absent here) on all host cores, rank 0 only.  Every step
    sorts the full configuration (the same 2^28 seeded keys as our arm, generated inside the
    oracle so that no library of the product is loaded), with the scratch the reference allocates
    per call made once outside the timed region."""
    if rank != 0:
        return
    if args.dtype != "u32":
        raise SystemExit("--impl reference runs the headline configuration (u32 keys) only")
    import oracle

    oracle.build()
    th = oracle.hardware_threads()
    n = args.n
    src = oracle.gen_u32_uniform(n, seed=1, threads=th)
    digest = input_digest(src)
    ws = oracle.RadixParWorkspace(n, 4)
    b = np.empty_like(src)
    for _ in range(args.warmup):
        np.copyto(b, src)
        ws.sort(b, threads=th)
    times = []
    for _ in range(args.steps):
        np.copyto(b, src)  # restore the input outside the timed region
        t0 = time.perf_counter()
        ws.sort(b, threads=th)
        times.append(time.perf_counter() - t0)
    if not _in_order(b):
        raise SystemExit("reference arm: output not sorted")
    ws.close()
    tot = sum(times)
    rate = n * args.steps / tot / 1e9
    line = {
        "metric": METRIC, "value": round(rate, 4), "unit": UNIT, "impl": "reference", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": round(tot / args.steps * 1e3, 4),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": args.dtype,
        "data": "synthetic (seeded PCG32 uniform keys)",
        "config": plain_config(n, "u32", world, digest),
        "residency": "host memory (the reference sorts managed host arrays)",
        "cpu_baseline": {"value": round(rate, 4), "unit": UNIT, "cores": th, "kind": "port",
                         "sample": f"the full {n}-key configuration every step; C++ restatement of "
                                   f"SortRadixPar (RadixSortLsdParallel.cs:145-232), 64 Ki work quanta, "
                                   f"{th} threads, scratch allocated once outside the timed region"},
        "e2e": {"value": round(rate, 4), "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------------------
def run_ours(args, rank: int, world: int, local_rank: int):
    import torch

    from hpcsharp_b200 import native, replicas

    dev = local_rank
    torch.cuda.set_device(dev)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist_mod

        dist_mod.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        dist = dist_mod

    n, dtype = args.n, args.dtype
    w = np.dtype(native.NP_OF[dtype]).itemsize
    P = w
    host = gen_keys(dtype, n, seed=1 + rank)
    tview = {4: torch.int32, 8: torch.int64}[w]
    src = torch.from_numpy(host.view({4: np.int32, 8: np.int64}[w])).to(f"cuda:{dev}")
    slots = [src.clone() for _ in range(max(1, args.slots))]
    ctx = native.Context(dev, pass_scheme=args.scheme)
    s = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{dev}")

    def step(i):
        ctx.sort_dev(slots[i % len(slots)], dtype=dtype)

    def restore(i):
        with torch.cuda.stream(s):
            slots[i % len(slots)].copy_(src)

    # warm-up
    for i in range(args.warmup):
        step(i)
        restore(i)
    ctx.synchronize()
    for i in range(len(slots)):
        restore(i)
    torch.cuda.synchronize()

    hbm, peak_kind = peaks()
    clocks = ClockSampler(dev)
    clocks.start()
    time.sleep(0.3)
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    ctx.profile(True)
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for i in range(args.steps):
        evs[i][0].record(s)
        step(i)
        evs[i][1].record(s)
        restore(i)
    ctx.synchronize()
    torch.cuda.synchronize()
    prof = ctx.profile_read()
    ctx.profile(False)
    total_ms = sum(a.elapsed_time(b) for a, b in evs)
    total_ms = replicas.max_over_ranks(total_ms, device=f"cuda:{dev}")
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()

    value = replicas.weak_scaling_gkeys(n, args.steps, world, total_ms)
    ms_per_step = total_ms / args.steps

    # roofline of the dominant kernel, the digit pass of whichever scheme ran (chunked:
    # profile class "onesweep", look-back: "lookback"; with float keys both kinds are launched
    # and the kind not chosen returns at once): algorithmic bytes per launch = one read + one
    # write of the keys = 2 * n * w
    chunked_ran = prof["onesweep"][1] >= prof["lookback"][1]
    os_launches, os_ms = prof["onesweep"] if chunked_ran else prof["lookback"]
    os_avg_ms = os_ms / max(1, os_launches)
    os_bytes = 2.0 * n * w
    achieved = os_bytes / (os_avg_ms / 1e3) / 1e9 if os_launches else None
    roof = {"kernel": "chunk_pass" if chunked_ran else "onesweep_pass (look-back)", "bound": "hbm", "achieved": round(achieved, 1) if achieved else None,
            "peak": hbm, "peak_kind": peak_kind, "unit": "GB/s",
            "frac": round(achieved / hbm, 4) if achieved else None,
            "traffic": read_traffic(dtype), "algorithmic_bytes_per_launch": os_bytes,
            "avg_launch_ms": round(os_avg_ms, 5), "launches": os_launches}
    sort_bytes = n * w * (1 + 2 * P)
    sort_achieved = sort_bytes / (ms_per_step / 1e3) / 1e9
    sort_roof = {"bytes_per_step": sort_bytes, "achieved": round(sort_achieved, 1), "peak": hbm,
                 "unit": "GB/s", "frac": round(sort_achieved / hbm, 4),
                 "kernels_ms_per_step": {k: round(v[1] / args.steps, 5) for k, v in prof.items() if v[0]}}
    launches = sum(v[0] for v in prof.values())

    # end to end through the host-array C ABI call, on a pageable host array (what a fixed .NET
    # array is: the library stages it through its pinned buffers) and on a pinned one
    e2e = e2e_pinned = None
    if not args.no_e2e:
        ksteps = args.e2e_steps or min(args.steps, 20)
        lib = native.load()
        fn = getattr(lib, f"hpcs_sort_{dtype}")

        def e2e_run(buf, api):
            np.copyto(buf, host)
            native.check(fn(ctx.handle, buf.ctypes.data, n))  # warm
            tot = 0.0
            for _ in range(ksteps):
                np.copyto(buf, host)
                if dist:
                    dist.barrier()
                t0 = time.perf_counter()
                native.check(fn(ctx.handle, buf.ctypes.data, n))
                tot += time.perf_counter() - t0
            tot = replicas.max_over_ranks(tot, device=f"cuda:{dev}")
            if not _in_order(buf):  # the last result must be in order
                raise RuntimeError("e2e result is not sorted")
            return {"value": round(n * ksteps * world / tot / 1e9, 4), "unit": UNIT,
                    "h2d_bytes_per_step": n * w, "d2h_bytes_per_step": n * w, "steps": ksteps,
                    "ms_per_step": round(tot / ksteps * 1e3, 3), "api": api}

        pageable = np.empty_like(host)
        e2e = e2e_run(pageable, f"hpcs_sort_{dtype} (host array in pageable memory, as a fixed .NET array)")
        del pageable
        pinned = torch.empty(n, dtype=tview, pin_memory=True)
        e2e_pinned = e2e_run(pinned.numpy().view(host.dtype), f"hpcs_sort_{dtype} (host array in pinned memory)")
        del pinned

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(dtype, n)

    if dist:
        dist.destroy_process_group()
    if rank == 0:
        line = {
            "metric": METRIC, "value": round(value, 4), "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": round(ms_per_step, 5), "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype,
            "data": "synthetic (seeded PCG32 uniform keys)",
            "config": plain_config(n, dtype, world, input_digest(host)),
            "residency": "device memory (value); host memory through the C ABI (e2e, e2e_pinned); "
                         "inputs restored between steps",
            "roofline": roof, "sort_roofline": sort_roof, "cpu_baseline": cpu, "e2e": e2e, "e2e_pinned": e2e_pinned,
            "gpu_launches": launches, "clocks": clk, "rank_mode": ctx.rank_mode,
        }
        print(json.dumps(line), flush=True)
    ctx.close()


def sort_bytes(n: int, w: int) -> int:
    """Algorithmic bytes of one plain sort: one histogram read + a read and a write per pass."""
    return n * w * (1 + 2 * w)


def run_batched(args, rank: int, world: int, local_rank: int, emit: bool = True):
    """65,536 arrays of mixed length and dtype: one graph-captured plan (the arrays binned by
    length class into the tuned warp- and block-level kernels) vs one plain sort call per array,
    same arrays, same device."""
    import torch

    from hpcsharp_b200 import native, workloads

    dev = local_rank
    torch.cuda.set_device(dev)
    lengths, dtypes = workloads.batched_lengths(
        count=args.arrays, target_total=None if args.literal else 250_000_000 * args.arrays // 65536, seed=4 + rank)
    bset = workloads.BatchedSet(lengths, dtypes, seed=1 + rank)
    tv = {4: (torch.int32, np.int32), 8: (torch.int64, np.int64)}
    pools, pristine = {}, {}
    for dt, host in bset.pools.items():
        w = host.dtype.itemsize
        pristine[dt] = torch.from_numpy(host.view(tv[w][1])).to(f"cuda:{dev}")
        pools[dt] = pristine[dt].clone()
    segs = []
    for dt, off, n in bset.items:
        w = np.dtype(workloads.datagen_dtype(dt)).itemsize
        segs.append(((pools[dt].data_ptr() + off * w, n), dt))
    ctx = native.Context(dev)
    s = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{dev}")

    def restore():
        with torch.cuda.stream(s):
            for dt in pools:
                pools[dt].copy_(pristine[dt])

    tuning = ctx.seg_tuning
    limits = native.seg_class_limits()

    def cls(n):
        for c, lim in enumerate(limits):
            if lim < 0 or n <= lim:
                return c

    variants_used = sorted({tuning[1 if dt in ("u64", "i64", "f64") else 0][cls(n)] for (_, n), dt in segs})
    plan = ctx.segplan(segs)
    for _ in range(max(1, args.warmup)):
        restore()
        plan.execute()
    ctx.synchronize()
    steps = max(1, min(args.steps, 20))
    tot = 0.0
    for _ in range(steps):
        restore()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        plan.execute()
        b.record(s)
        ctx.synchronize()
        tot += a.elapsed_time(b)
    batched_ms = tot / steps
    # the same arrays, one plain sort call each
    lib = native.load()
    fns = {dt: getattr(lib, f"hpcs_sort_{dt}_dev") for dt in set(dtypes)}
    plain_ms = []
    for _ in range(2):
        restore()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(s)
        for (ptr, n), dt in segs:
            native.check(fns[dt](ctx.handle, ptr, n, None))
        b.record(s)
        ctx.synchronize()
        plain_ms.append(a.elapsed_time(b))
    plain_ms = min(plain_ms)
    # spot check: every 997th array is in order
    for i in range(0, len(segs), 997):
        dt, off, n = bset.items[i]
        t = pools[dt][off:off + n].cpu().numpy().view(workloads.datagen_dtype(dt))
        if not _in_order(t):
            raise RuntimeError(f"batched array {i} ({dt}, n={n}) is not sorted")
    plan.close()
    ctx.close()
    nbytes = int(sum(sort_bytes(int(n), np.dtype(workloads.datagen_dtype(dt)).itemsize)
                     for n, dt in zip(lengths, dtypes)))
    hbm, peak_kind = peaks()
    out = {
        "workload": "batched segmented sort", "arrays": len(segs), "total_keys": bset.total_keys,
        "length_distribution": "log-uniform [32, 2^20]" + ("" if args.literal else ", scaled to ~250M keys"),
        "dtypes": list(workloads.BATCH_DTYPES), "batched_ms": round(batched_ms, 3),
        "batched_gkeys_s": round(bset.total_keys / (batched_ms / 1e3) / 1e9, 3),
        "plain_per_array_ms": round(plain_ms, 3),
        "plain_per_array_gkeys_s": round(bset.total_keys / (plain_ms / 1e3) / 1e9, 3),
        "speedup_vs_per_array": round(plain_ms / batched_ms, 2),
        "roofline": {"bytes": nbytes, "achieved": round(nbytes / (batched_ms / 1e3) / 1e9, 1), "peak": hbm,
                     "peak_kind": peak_kind, "unit": "GB/s",
                     "frac": round(nbytes / (batched_ms / 1e3) / 1e9 / hbm, 4)},
        "launches": "1 graph (one persistent launch per kernel variant in use, as concurrent branches) vs "
                    + str(len(segs)) + " plain sort calls",
        "seg_tuning": tuning, "variants_used": variants_used,
    }
    if emit and rank == 0:
        line = {"metric": METRIC, "value": out["batched_gkeys_s"], "unit": UNIT, "n_gpus": world,
                "steps": steps, "warmup": args.warmup, "ms_per_step": out["batched_ms"], "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "mixed u32/i32/f32/u64",
                "data": "synthetic (seeded)", "config": {"workload": out["workload"], "arrays": len(segs)},
                "batched": out}
        print(json.dumps(line), flush=True)
    return out


def _pct(v, q):
    return float(np.percentile(np.asarray(v), q)) if len(v) else None


def run_served(args, rank: int, world: int, local_rank: int, emit: bool = True):
    """Serving loop vs the plain form on the same GPU: the same seeded trace of sort and top-k
    requests arrives as a Poisson process; the server (continuous batching, HBM admission,
    coalescing of small requests) is compared with plain synchronous calls that take the
    requests one at a time in arrival order.  Every served result is compared byte for byte
    with the plain result."""
    import threading

    import torch

    from hpcsharp_b200 import datagen, native, workloads

    dev = local_rank
    torch.cuda.set_device(dev)
    reqs, gaps = workloads.serving_trace(count=args.requests, seed=9 + rank)
    npdt = {dt: workloads.datagen_dtype(dt) for dt in workloads.SERVE_DTYPES}
    # pinned host buffers for every request's input and output
    inputs, outs_served, outs_plain = [], [], []
    for i, (op, dt, n, k) in enumerate(reqs):
        w = np.dtype(npdt[dt]).itemsize
        pin = torch.empty(n * w, dtype=torch.uint8, pin_memory=True).numpy().view(npdt[dt])
        datagen_out = datagen.by_name(dt, n, seed=1000 + i)
        np.copyto(pin, datagen_out)
        inputs.append(pin)
        m = n if op == "sort" else k
        outs_served.append(torch.empty(m * w, dtype=torch.uint8, pin_memory=True).numpy().view(npdt[dt]))
        outs_plain.append(np.empty(m, dtype=npdt[dt]))
    total_keys = sum(n for _, _, n, _ in reqs)
    ctx = native.Context(dev)

    def plain_call(i):
        op, dt, n, k = reqs[i]
        if op == "sort":
            np.copyto(outs_plain[i], inputs[i])
            ctx.sort(outs_plain[i])
        else:
            outs_plain[i][...] = ctx.topk_largest(inputs[i], k)

    # plain service time of every request (also warms the plain path)
    service = []
    for i in range(len(reqs)):
        t0 = time.perf_counter()
        plain_call(i)
        service.append(time.perf_counter() - t0)
    mean_service = float(np.mean(service))
    budget = 64 << 30
    server = native.Server(dev, slots=4, hbm_budget_bytes=budget, coalesce_max_keys=1 << 17)
    for i in range(min(8, len(reqs))):  # warm the server path
        server.wait(server.submit(reqs[i][0], inputs[i], outs_served[i], reqs[i][3]))

    points = []
    for load in (float(x) for x in args.loads.split(",")):
        rate = load / mean_service  # requests per second
        arrivals = np.cumsum(gaps) / rate
        # served: a client thread submits at the arrival times
        tickets = [None] * len(reqs)
        t_base = time.perf_counter() + 0.05

        def client():
            for i, t_arr in enumerate(arrivals):
                d = t_base + t_arr - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets[i] = server.submit(reqs[i][0], inputs[i], outs_served[i], reqs[i][3])

        th = threading.Thread(target=client)
        th.start()
        th.join()
        infos = [server.wait(t) for t in tickets]
        lat = [(x["done_ns"] - x["submit_ns"]) / 1e6 for x in infos]
        span = (max(x["done_ns"] for x in infos) - min(x["submit_ns"] for x in infos)) / 1e9
        for i in range(len(reqs)):
            if not np.array_equal(outs_served[i].view(np.uint8), outs_plain[i].view(np.uint8)):
                raise RuntimeError(f"served result {i} differs from the plain result")
        # plain: one request at a time, each starting at max(arrival, previous completion)
        t_base = time.perf_counter() + 0.01
        plat = []
        t_first = None
        for i, t_arr in enumerate(arrivals):
            d = t_base + t_arr - time.perf_counter()
            if d > 0:
                time.sleep(d)
            if t_first is None:
                t_first = time.perf_counter()
            plain_call(i)
            plat.append((time.perf_counter() - (t_base + t_arr)) * 1e3)
        pspan = time.perf_counter() - t_first
        points.append({
            "offered_load": load, "rate_req_s": round(rate, 1),
            "served": {"p50_ms": round(_pct(lat, 50), 3), "p99_ms": round(_pct(lat, 99), 3),
                       "gkeys_s": round(total_keys / span / 1e9, 3),
                       "coalesced": int(sum(x["coalesced"] for x in infos))},
            "plain": {"p50_ms": round(_pct(plat, 50), 3), "p99_ms": round(_pct(plat, 99), 3),
                      "gkeys_s": round(total_keys / pspan / 1e9, 3)},
        })
    st = server.stats()
    server.close()
    ctx.close()
    out = {
        "workload": "served sort/top-k requests", "requests_per_rate": len(reqs), "total_keys": total_keys,
        "mix": "70% sort / 30% top-k (k in {10, 1000, 100000}), n log-uniform [1K, 64M], u32/i32/f32/u64",
        "plain_mean_service_ms": round(mean_service * 1e3, 3), "hbm_budget_bytes": budget,
        "arena_peak_bytes": st["arena_peak"], "sweep": points, "results": "every served result == plain result",
        "host_buffers": "pinned",
    }
    best = max(points, key=lambda p: p["served"]["gkeys_s"])
    if emit and rank == 0:
        line = {"metric": METRIC, "value": best["served"]["gkeys_s"], "unit": UNIT, "n_gpus": world,
                "steps": len(points), "warmup": 8, "ms_per_step": None, "higher_is_better": True,
                "scaling": "weak", "vs_baseline": None, "dtype": "mixed u32/i32/f32/u64",
                "data": "synthetic (seeded)", "config": {"workload": out["workload"]}, "served": out}
        print(json.dumps(line), flush=True)
    return out


def run_configs(args, rank: int, world: int, local_rank: int):
    """Every plain-sort and key+index configuration, device-resident: the input restored before
    each of K sorts (outside the CUDA events), Gkeys/s and the fraction of the bytes-moved
    roofline N*w*(1 + 2P) (+ 2P*N*4 for an index payload)."""
    import torch

    from hpcsharp_b200 import datagen, native

    if rank != 0:
        return
    dev = local_rank
    torch.cuda.set_device(dev)
    hbm, peak_kind = peaks()
    ctx = native.Context(dev)
    s = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{dev}")
    steps = max(1, min(args.steps, 10))
    cfgs = [
        ("C1 u32 uniform (PCG32 stream)", "u32", 10_000_000, lambda n: datagen.u32_pcg32_stream(n, 1), False),
        ("C2 u32 uniform", "u32", 1 << 28, lambda n: datagen.u32_uniform(n, 1), False),
        ("C2 i32 normal(0, 2^20)", "i32", 1 << 28, lambda n: datagen.i32_normal(n, 1), False),
        ("C2 f32 normal(0,1) + specials", "f32", 1 << 28, lambda n: datagen.f32_normal_special(n, 1), False),
        ("C2 u64 uniform", "u64", 1 << 27, lambda n: datagen.u64_uniform(n, 1), False),
        ("C2 u64 AND of 3 uniform", "u64", 1 << 27, lambda n: datagen.u64_and3(n, 1), False),
        ("C3 u64 Zipf(1.1) keys + u32 index", "u64", 200_000_000, lambda n: datagen.u64_zipf(n, 1), True),
        ("C3 f64 normal keys + i32 index", "f64", 100_000_000, lambda n: datagen.f64_normal(n, 1), True),
    ]
    rows = []
    for name, dt, n, gen, pairs in cfgs:
        host = gen(n)
        w = host.dtype.itemsize
        P = w
        tv = torch.int32 if w == 4 else torch.int64
        pristine = torch.from_numpy(host.view(np.int32 if w == 4 else np.int64)).to(f"cuda:{dev}")
        buf = pristine.clone()
        vals = torch.empty(n, dtype=torch.int32, device=f"cuda:{dev}") if pairs else None
        iota = torch.arange(n, dtype=torch.int32, device=f"cuda:{dev}") if pairs else None

        def restore():
            with torch.cuda.stream(s):
                buf.copy_(pristine)
                if pairs:
                    vals.copy_(iota)

        def sort():
            if pairs:
                ctx.sort_pairs_dev(buf, vals, dtype=dt, stream=ctx.stream)
            else:
                ctx.sort_dev(buf, dtype=dt, stream=ctx.stream)

        for _ in range(max(3, args.warmup)):
            restore()
            sort()
        ctx.synchronize()
        tot = 0.0
        for _ in range(steps):
            restore()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            sort()
            b.record(s)
            ctx.synchronize()
            tot += a.elapsed_time(b)
        ms = tot / steps
        nbytes = n * w * (1 + 2 * P) + (2 * P * n * 4 if pairs else 0)
        achieved = nbytes / (ms / 1e3) / 1e9
        o = buf[:1 << 20].cpu().numpy().view(host.dtype)
        if not _in_order(o):
            raise RuntimeError(f"{name}: result not in order")
        rows.append({"config": name, "dtype": dt, "n": n, "pairs": pairs, "ms": round(ms, 3),
                     "gkeys_s": round(n / (ms / 1e3) / 1e9, 3), "algorithmic_bytes": nbytes,
                     "achieved_gbs": round(achieved, 1), "roofline_frac": round(achieved / hbm, 4),
                     "l2": "inputs larger than L2" if n * w > (126 << 20) else "input fits in L2 (not graded)"})
        del pristine, buf, vals, iota
        torch.cuda.empty_cache()
    ctx.close()
    print(json.dumps({"metric": METRIC, "workload": "configs", "unit": UNIT, "peak": hbm, "peak_kind": peak_kind,
                      "steps": steps, "rows": rows}), flush=True)


def run_kernels(args, rank: int, world: int, local_rank: int):
    """The path's other entry points on device-resident keys, CUDA events on the context's
    stream, input restored before each call outside the events, mean of up to 10 calls after 3
    warm-ups: radix top-k (the k largest, out of place) of 2^28 u32 keys for k in {10, 1000,
    100000}; SelectTopK in place (select + stable 3-way partition) of the same keys; the
    counting sorts of 2^28 u8 and u16 keys.  Roofline bytes: top-k one read of the keys (its
    minimum), SelectTopK the select's histogram read plus the partition's read and write,
    counting sort one read (histogram) plus one write (fill)."""
    import torch

    from hpcsharp_b200 import datagen, native

    if rank != 0:
        return
    dev = local_rank
    torch.cuda.set_device(dev)
    hbm, peak_kind = peaks()
    ctx = native.Context(dev)
    s = torch.cuda.ExternalStream(ctx.stream, device=f"cuda:{dev}")
    steps = max(1, min(args.steps, 10))
    n = 1 << 28
    rng = np.random.default_rng(5)
    u32 = torch.from_numpy(datagen.u32_uniform(n, 1).view(np.int32)).to(f"cuda:{dev}")
    u8 = torch.from_numpy(rng.integers(0, 256, n, dtype=np.uint8)).to(f"cuda:{dev}")
    u16 = torch.from_numpy(rng.integers(0, 1 << 16, n, dtype=np.uint16).view(np.int16)).to(f"cuda:{dev}")
    out = torch.empty(100_000, dtype=torch.int32, device=f"cuda:{dev}")
    cases = []
    for k in (10, 1000, 100_000):
        cases.append((f"top-k largest, k={k}", "u32", u32, False,
                      lambda t, k=k: ctx.topk_largest_dev(t, k, out[:k], dtype="u32", stream=ctx.stream), n * 4))
    cases.append(("SelectTopK in place, k=n/2", "u32", u32, True,
                  lambda t: ctx.select_topk_dev(t, n // 2, dtype="u32", stream=ctx.stream), 3 * n * 4))
    cases.append(("counting sort", "u8", u8, True, lambda t: ctx.sort_dev(t, dtype="u8", stream=ctx.stream), 2 * n))
    cases.append(("counting sort", "u16", u16, True, lambda t: ctx.sort_dev(t, dtype="u16", stream=ctx.stream),
                  2 * n * 2))
    rows = []
    for name, dt, src, in_place, call, nbytes in cases:
        buf = src.clone() if in_place else src
        tot = 0.0
        for i in range(3 + steps):
            if in_place:
                with torch.cuda.stream(s):
                    buf.copy_(src)
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record(s)
            call(buf)
            b.record(s)
            ctx.synchronize()
            if i >= 3:
                tot += a.elapsed_time(b)
        ms = tot / steps
        gbs = nbytes / (ms / 1e3) / 1e9
        rows.append({"op": name, "dtype": dt, "n": n, "ms": round(ms, 4), "gkeys_s": round(n / (ms / 1e3) / 1e9, 2),
                     "roofline_bytes": nbytes, "achieved_gbs": round(gbs, 1), "roofline_frac": round(gbs / hbm, 4)})
        if in_place and buf is not src:
            del buf
    srt = u8.clone()
    ctx.sort_dev(srt, dtype="u8", stream=ctx.stream)
    ctx.synchronize()
    head = srt[:1 << 20].cpu().numpy()
    if not np.all(head[1:] >= head[:-1]):
        raise RuntimeError("counting sort result not in order")
    ctx.close()
    print(json.dumps({"metric": METRIC, "workload": "kernels", "unit": UNIT, "peak": hbm, "peak_kind": peak_kind,
                      "steps": steps, "rows": rows}), flush=True)


def run_sharded(args, rank: int, world: int, local_rank: int):
    """The sharded sort of one array of world x n keys (n per rank, weak scaling): every step
    partitions, exchanges (NCCL all-to-all), sorts and rebalances; CUDA events on the current
    stream around each step (host synchronisations of the exchange sizes included), max over
    ranks.  Also times the partition kernel alone into 8 parts (its roofline: one read and one
    write of the keys per launch)."""
    import datetime

    import torch
    import torch.distributed as dist

    from hpcsharp_b200 import native, replicas, sharded

    dev = local_rank
    torch.cuda.set_device(dev)
    if "MASTER_ADDR" not in os.environ:
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(29400 + os.getpid() % 500))
    dist.init_process_group("nccl", rank=rank, world_size=world, timeout=datetime.timedelta(seconds=120),
                            device_id=torch.device(f"cuda:{dev}"))
    n, dtype = args.n, args.dtype
    w = np.dtype(native.NP_OF[dtype]).itemsize
    host = gen_keys(dtype, n, seed=1 + rank)
    keys = torch.from_numpy(host.view({4: np.int32, 8: np.int64}[w])).to(f"cuda:{dev}")
    ctx = native.Context(dev)
    ops = sharded.DeviceOps(ctx, dtype)
    for _ in range(max(3, args.warmup)):
        out, _ = sharded.sort_sharded(keys, ops=ops)
    torch.cuda.synchronize()
    steps = max(1, min(args.steps, 10))
    ctx.profile(True)
    tot = 0.0
    for _ in range(steps):
        dist.barrier()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        out, _ = sharded.sort_sharded(keys, ops=ops)
        b.record()
        torch.cuda.synchronize()
        tot += a.elapsed_time(b)
    prof = ctx.profile_read()
    ctx.profile(False)
    tot = replicas.max_over_ranks(tot, device=f"cuda:{dev}")
    ok = _in_order(out[:1 << 20].cpu().numpy().view(host.dtype)) and out.numel() == n
    # the partition kernel alone, 8 parts, splitters from a sorted sample of the keys
    parts = 8
    stream = native.torch_stream()
    samp = keys[torch.randint(0, n, (4096,), device=f"cuda:{dev}")].contiguous()
    idx = torch.arange(4096, dtype=torch.int32, device=f"cuda:{dev}")
    ctx.sort_pairs_dev(samp, idx, dtype=dtype, stream=stream)
    pick = torch.tensor([(j * 4096) // parts for j in range(1, parts)], device=f"cuda:{dev}")
    sk = samp[pick].contiguous()
    sg = torch.zeros(parts - 1, dtype=torch.int64, device=f"cuda:{dev}")
    ko = torch.empty_like(keys)
    cnt = torch.empty(parts, dtype=torch.int64, device=f"cuda:{dev}")
    for _ in range(3):
        ctx.shard_partition_dev(keys, None, 0, sk, sg, parts, ko, None, cnt, dtype=dtype, stream=stream)
    torch.cuda.synchronize()
    pt = []
    for _ in range(steps):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        ctx.shard_partition_dev(keys, None, 0, sk, sg, parts, ko, None, cnt, dtype=dtype, stream=stream)
        b.record()
        torch.cuda.synchronize()
        pt.append(a.elapsed_time(b))
    part_ms = statistics.median(pt)
    hbm, peak_kind = peaks()
    part_gbs = 2.0 * n * w / (part_ms / 1e3) / 1e9
    dist.destroy_process_group()
    if rank == 0:
        print(json.dumps({
            "metric": "Gkeys/s, sharded sort of one array across ranks", "workload": "sharded",
            "value": round(n * world * steps / (tot / 1e3) / 1e9, 4), "unit": UNIT, "n_gpus": world,
            "steps": steps, "ms_per_step": round(tot / steps, 4), "scaling": "weak", "dtype": dtype,
            "config": {"keys_per_rank": n, "dtype": dtype, "balance": True, "samples_per_rank": 1024},
            "sorted": bool(ok),
            "kernels_ms_per_step": {k: round(v[1] / steps, 4) for k, v in prof.items() if v[0]},
            "partition_8_parts": {"ms": round(part_ms, 4), "achieved_gbs": round(part_gbs, 1),
                                  "algorithmic_bytes": 2 * n * w, "peak": hbm, "peak_kind": peak_kind,
                                  "frac": round(part_gbs / hbm, 4), "counts": cnt.cpu().tolist()},
        }), flush=True)
    ctx.close()


def main():
    args = parse()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.workload == "batched":
        run_batched(args, rank, world, local_rank)
        return
    if args.workload == "served":
        run_served(args, rank, world, local_rank)
        return
    if args.workload == "configs":
        run_configs(args, rank, world, local_rank)
        return
    if args.workload == "sharded":
        run_sharded(args, rank, world, local_rank)
        return
    if args.workload == "kernels":
        run_kernels(args, rank, world, local_rank)
        return
    run_ours(args, rank, world, local_rank)


if __name__ == "__main__":
    main()

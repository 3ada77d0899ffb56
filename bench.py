"""Benchmark of the LNT B200 hot path.

Default workload (one JSON line on rank 0): the sparse merge under index
permutation c(i,j,k,l) = a(i,j,k,l) + b(l,k,j,i), order-4 SparseMIA with dims
512^4 (36-bit linear keys), 2^26 non-zeros per operand, uniform random
coordinates (drawn with replacement), float64 values uniform[-1, 1], both
operands unsorted, so the reference takes SparseMIA::sortMerge: re-key A into
B's order, concatenate, sort, collect duplicates with +.

A "step" is one such merge.  `value` = merged input non-zeros per second with
the operands resident in HBM; `e2e` = the same through the C ABI from pinned
host buffers, host->device copies of both operands and the device->host copy
of the result inside the timed region.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

With --gpus N > 1 (under torchrun) every rank merges its own independent
operand pair (no collective on the data path: weak scaling, replicas).
"""
from __future__ import annotations

import argparse
import contextlib
import json
import os
import statistics
import sys
import threading
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "sparse contraction products/s & %HBM peak; FP64-accurate dense TFLOP/s"
DIMS = [512, 512, 512, 512]
NNZ = 1 << 26
MAX_KEY = 512 ** 4
INDEX_ORDER = [3, 2, 1, 0]  # c(i,j,k,l) = a(i,j,k,l) + b(l,k,j,i)
WORKLOAD = ("sparse merge c(i,j,k,l)=a(i,j,k,l)+b(l,k,j,i): order-4 SparseMIA dims 512^4, "
            "2^26 nnz per operand, uniform coordinates, f64 values U[-1,1], both unsorted (sortMerge: "
            "re-key A to {3,2,1,0}, concatenate, radix-sort the 2^27 (u64,f64) pairs, collect duplicates)")
IMPLEMENTATION = ("bucket histogram (A re-keyed on the fly), two 8-bit onesweep passes over the top 15 key bits, "
                  "per-bucket shared-memory sort with the duplicate fold fused")
HBM_FALLBACK_GBS = 6650.0
L2_NOTE = "inputs (2 GiB) and sort buffers larger than the 126 MB L2; no flush needed"


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


def tuned_value(key: str):
    """A value the autotuner compiled into the library (libnt_b200/csrc/lnt_tuned.json)."""
    f = ROOT / "libnt_b200" / "csrc" / "lnt_tuned.json"
    return json.loads(f.read_text()).get(key) if f.exists() else None


def profile_traffic(name: str, key: str = "traffic_bytes_per_pair"):
    """Per-unit DRAM traffic of a kernel from the committed ncu summary
    (line '<key>: X'), or None."""
    f = ROOT / "profiles" / f"{name}.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.strip().startswith(key + ":"):
            try:
                return float(line.split(":", 1)[1].strip().split()[0])
            except ValueError:
                return None
    return None


# ---------------------------------------------------------------------------
# clocks during the timed region (NVML)
# ---------------------------------------------------------------------------
class ClockSampler:
    REASONS = {0x1: "gpu_idle", 0x2: "applications_clocks_setting", 0x4: "sw_power_cap", 0x8: "hw_slowdown",
               0x20: "sync_boost", 0x40: "sw_thermal_slowdown", 0x80: "hw_thermal_slowdown",
               0x100: "hw_power_brake_slowdown", 0x200: "display_clock_setting"}

    def __init__(self, device_index: int, period_s: float = 0.02):
        self.samples = []
        self.reasons = 0
        self.max_mhz = None
        self._stop = threading.Event()
        self._period = period_s
        self._h = None
        try:
            import pynvml
            pynvml.nvmlInit()
            self._nvml = pynvml
            self._h = pynvml.nvmlDeviceGetHandleByIndex(device_index)
            self.max_mhz = pynvml.nvmlDeviceGetMaxClockInfo(self._h, pynvml.NVML_CLOCK_SM)
        except Exception:
            self._h = None

    def _run(self):
        n = self._nvml
        while not self._stop.is_set():
            try:
                self.samples.append(n.nvmlDeviceGetClockInfo(self._h, n.NVML_CLOCK_SM))
                try:
                    r = n.nvmlDeviceGetCurrentClocksEventReasons(self._h)
                except AttributeError:
                    r = n.nvmlDeviceGetCurrentClocksThrottleReasons(self._h)
                self.reasons |= int(r)
            except Exception:
                pass
            time.sleep(self._period)

    def __enter__(self):
        if self._h is not None:
            self._t = threading.Thread(target=self._run, daemon=True)
            self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        if self._h is not None:
            self._t.join()

    def summary(self):
        if self._h is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvml unavailable"]}
        reasons = [v for k, v in self.REASONS.items() if self.reasons & k and k != 0x1]
        return {"sm_mhz": statistics.median(self.samples) if self.samples else None, "sm_max_mhz": self.max_mhz,
                "reasons": reasons, "samples": len(self.samples)}


# ---------------------------------------------------------------------------
# distributed plumbing
# ---------------------------------------------------------------------------
def dist_setup(n_gpus: int):
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime
        import torch.distributed as dist
        torch.cuda.set_device(local)
        if not dist.is_initialized():
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
    elif torch.cuda.is_available():
        torch.cuda.set_device(0)
    return world, rank, local


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x: float, world: int) -> float:
    """Largest per-rank value (step time): the job is as slow as its slowest rank."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    dev = "cpu" if dist.get_backend() == "gloo" else "cuda"
    t = torch.tensor([x], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(units_per_rank: int, world: int, ms_max: float) -> float:
    """Whole-job throughput of `world` replicas: all ranks' units over the slowest rank's time."""
    return units_per_rank * world / (ms_max * 1e-3)


# ---------------------------------------------------------------------------
# CPU side: the reference's own kernels (oracle/_ref) or the restatement
# ---------------------------------------------------------------------------
def cpu_merge_sample(n_per_operand: int, seed: int = 0):
    """One reference sortMerge on a bounded sample; returns (seconds, kind)."""
    import oracle
    rng = np.random.default_rng(seed)
    ak = rng.integers(0, MAX_KEY, n_per_operand, dtype=np.uint64)
    bk = rng.integers(0, MAX_KEY, n_per_operand, dtype=np.uint64)
    av = rng.uniform(-1, 1, n_per_operand)
    bv = rng.uniform(-1, 1, n_per_operand)
    kind = "reference" if oracle.ref_available() else "port"
    t0 = time.perf_counter()
    if kind == "reference":
        # SparseMIA::sortMerge: change_linIdx_sequence (reference re-key), concatenate,
        # collect_duplicates = reference radix sort + fold (restated)
        ka = oracle.ref_rekey(ak, DIMS, [0, 1, 2, 3], [3, 2, 1, 0])
        k = np.concatenate([ka, bk])
        v = np.concatenate([av, bv])
        k, v = oracle.ref_radix_sort(k, v, MAX_KEY)
        oracle.collect_duplicates(k, v)
    else:
        ka = oracle.rekey(ak, DIMS, [0, 1, 2, 3], [3, 2, 1, 0])
        k, v = oracle.sort_pairs(np.concatenate([ka, bk]), np.concatenate([av, bv]))
        oracle.collect_duplicates(k, v)
    return time.perf_counter() - t0, kind


CPU_SAMPLE = 1 << 23  # per operand: 2^24 pairs, ~1/8 of the workload


def _host_cores() -> int:
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


# ---- reference arm: the full merge per step, spread over the host cores -----
# The reference is single-threaded (its OpenMP is commented out).  To use every
# host core on the same workload, each step runs one complete 2 x 2^26
# sortMerge: the reference's own re-key on slices of A, then the key range is
# cut into one part per worker and each worker sorts its part with the
# reference's own MSD radix sort and folds it with the restated
# collect_duplicates.  Parts are independent (equal keys share a part), so this
# is the same sort and fold as one sortMerge, with the top of the MSD
# recursion's bucket split done by key range.
_REF = {}


def _ref_attach(folder: str, n: int):
    import oracle
    oracle.ref_available()
    for name, dt in (("ak", np.uint64), ("av", np.float64), ("bk", np.uint64), ("bv", np.float64),
                     ("ka", np.uint64)):
        _REF[name] = np.memmap(os.path.join(folder, name), dtype=dt, mode="r+", shape=(n,))


def _ref_rekey_slice(bounds):
    import oracle
    lo, hi = bounds
    if oracle.ref_available():
        _REF["ka"][lo:hi] = oracle.ref_rekey(_REF["ak"][lo:hi], DIMS, [0, 1, 2, 3], INDEX_ORDER)
    else:
        _REF["ka"][lo:hi] = oracle.rekey(_REF["ak"][lo:hi], DIMS, [0, 1, 2, 3], INDEX_ORDER)
    return 0


def _ref_sort_part(bounds):
    import oracle
    lo, hi = bounds
    ka, bk = _REF["ka"], _REF["bk"]
    ma = (ka >= lo) & (ka < hi)
    mb = (bk >= lo) & (bk < hi)
    k = np.concatenate([ka[ma], bk[mb]])
    v = np.concatenate([_REF["av"][ma], _REF["bv"][mb]])
    if oracle.ref_available():
        k, v = oracle.ref_radix_sort(k, v, MAX_KEY)
    else:
        k, v = oracle.sort_pairs(k, v)
    ck, _ = oracle.collect_duplicates(k, v)
    return int(ck.size)


def run_reference(args):
    """The reference's own CPU path (re-key, MSD radix sort, collect) for the
    full workload on all host cores; see the comment above _REF."""
    import concurrent.futures as cf
    import multiprocessing as mp
    import shutil
    import tempfile
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    workers = _host_cores()
    n = NNZ
    folder = tempfile.mkdtemp(prefix="lnt_ref_", dir="/dev/shm" if os.path.isdir("/dev/shm") else None)
    try:
        rng = np.random.default_rng(4321)
        for name in ("ak", "bk"):
            m = np.memmap(os.path.join(folder, name), dtype=np.uint64, mode="w+", shape=(n,))
            m[:] = rng.integers(0, MAX_KEY, n, dtype=np.uint64)
            m.flush()
        for name in ("av", "bv"):
            m = np.memmap(os.path.join(folder, name), dtype=np.float64, mode="w+", shape=(n,))
            m[:] = rng.uniform(-1, 1, n)
            m.flush()
        np.memmap(os.path.join(folder, "ka"), dtype=np.uint64, mode="w+", shape=(n,)).flush()
        slices = [(n * w // workers, n * (w + 1) // workers) for w in range(workers)]
        parts = [(MAX_KEY * w // workers, MAX_KEY * (w + 1) // workers) for w in range(workers)]
        times = []
        out_nnz = 0
        import oracle
        kind = "reference" if oracle.ref_available() else "port"
        with cf.ProcessPoolExecutor(max_workers=workers, mp_context=mp.get_context("spawn"),
                                    initializer=_ref_attach, initargs=(folder, n)) as pool:
            list(pool.map(_warm_worker, range(workers)))  # imports and library loads outside the timing
            for i in range(args.warmup + args.steps):
                t0 = time.perf_counter()
                list(pool.map(_ref_rekey_slice, slices))
                out_nnz = sum(pool.map(_ref_sort_part, parts))
                t = time.perf_counter() - t0
                if i >= args.warmup:
                    times.append(t)
    finally:
        shutil.rmtree(folder, ignore_errors=True)
    t = statistics.median(times)
    rate = 2 * n / t
    sample = (f"the full workload every step: one 2 x 2^26 sortMerge, A re-keyed in {workers} slices, then "
              f"{workers} key ranges each sorted by "
              + ("the reference's MSD radix sort" if kind == "reference" else "the restated sort")
              + " and folded by the restated collect_duplicates, one worker process per host core")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "nnz/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nnz_per_operand": NNZ, "l2": L2_NOTE},
            "parallelism": f"{workers} host processes over key ranges of one merge",
            "output_nnz": out_nnz,
            "cpu_baseline": {"value": rate, "unit": "nnz/s", "cores": workers, "kind": kind, "sample": sample},
            "e2e": {"value": rate, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


def _warm_worker(_):
    import oracle
    oracle.ref_available()
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def oracle_window_check(ak, av, bk, bv, out_k, out_v, windows=4, width=1 << 24, seed=99):
    """Checks the device merge against the oracle on key windows: the pairs of
    A (re-keyed by the oracle) and B whose keys fall in [lo, lo + width) are
    sorted and folded on the host, and must equal the device output's slice
    for that range (keys exact, values within 1e-12 of the sum of |addends|).
    The first window starts at key 0, so the position-0 rule of
    collect_duplicates is checked as well.  Raises on a mismatch."""
    import oracle
    ak, av, bk, bv = (t.cpu().numpy() for t in (ak, av, bk, bv))
    ka = oracle.rekey(ak.view(np.uint64), DIMS, [0, 1, 2, 3], INDEX_ORDER)
    bk = bk.view(np.uint64)
    gk = out_k.cpu().numpy().view(np.uint64)
    gv = out_v.cpu().numpy()
    rng = np.random.default_rng(seed)
    los = [0] + [int(x) for x in rng.integers(1, MAX_KEY - width, windows - 1)]
    checked = 0
    for lo in los:
        hi = lo + width
        ma = (ka >= lo) & (ka < hi)
        mb = (bk >= lo) & (bk < hi)
        k, v = oracle.sort_pairs(np.concatenate([ka[ma], bk[mb]]), np.concatenate([av[ma], bv[mb]]))
        ek, ev, ea = oracle.collect_duplicates(k, v, with_abs=True)
        i0, i1 = np.searchsorted(gk, lo), np.searchsorted(gk, hi)
        if not np.array_equal(gk[i0:i1], ek):
            raise RuntimeError(f"merge output keys differ from the oracle in key window [{lo}, {hi})")
        if not np.all(np.abs(gv[i0:i1] - ev) <= 1e-12 * ea):
            raise RuntimeError(f"merge output values differ from the oracle in key window [{lo}, {hi})")
        checked += ek.size
    return {"windows": len(los), "window_keys": width, "output_entries_checked": checked, "ok": True}


E2E_LANES = 3  # copy/merge streams of the end-to-end measurement


def run_ours(args):
    import torch

    import libnt_b200 as L

    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(1234 + rank)
    na = nb = 1 << args.nnz_log2
    ak = torch.randint(0, MAX_KEY, (na,), generator=g, device=dev, dtype=torch.int64)
    bk = torch.randint(0, MAX_KEY, (nb,), generator=g, device=dev, dtype=torch.int64)
    av = torch.rand(na, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    bv = torch.rand(nb, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    spec = L.RekeySpec.make(DIMS, [0, 1, 2, 3], [3, 2, 1, 0])  # sortMerge, |A| == |B|: A to B's order
    n = na + nb
    out_k = torch.empty(n, dtype=torch.int64, device=dev)
    out_v = torch.empty(n, dtype=torch.float64, device=dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    ws = L.workspace(L.sort_reduce_workspace(na, nb, MAX_KEY), dev)

    def step():
        L.sort_reduce(ak, av, bk, bv, max_key=MAX_KEY, a_rekey=spec, out_keys=out_k, out_vals=out_v, count=cnt,
                      ws=ws, sync=False)

    stream = torch.cuda.current_stream()
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    assert L.device_status() == 0, "device-side wait expired during warm-up"

    # ---- device-resident timing -------------------------------------------
    L.profile_reset()
    L.profile_enable(True)
    launches0 = L.launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    sampler = ClockSampler(local if world > 1 else torch.cuda.current_device())
    barrier(world)
    torch.cuda.synchronize()
    with sampler:
        e0.record(stream)
        for _ in range(args.steps):
            step()
        e1.record(stream)
        torch.cuda.synchronize()
    barrier(world)
    launches = L.launch_count() - launches0
    L.profile_enable(False)
    ms = e0.elapsed_time(e1) / args.steps
    ms = max_over_ranks(ms, world)
    value = job_throughput(n, world, ms)
    kernels = {}
    for name in ("sort_hist", "sort_onesweep", "bucket_sort_collect", "collect_lead", "collect",
                 "sort_hist_fallback", "sort_onesweep_fallback", "collect_lead_fallback", "collect_fallback"):
        t, c = L.profile_query(name)
        kernels[name] = {"ms_total": t, "launches": c}
    L.profile_reset()
    n_out = int(cnt.item())
    assert L.device_status() == 0, "device-side wait expired during timing"
    check = oracle_window_check(ak, av, bk, bv, out_k[:n_out], out_v[:n_out]) if rank == 0 else None

    if args.no_e2e:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "nnz/s", "ms_per_step": ms,
                              "nnz_per_operand": na, "kernels": kernels}), flush=True)
        return 0

    # ---- end-to-end through the C ABI from pinned host buffers ------------
    # Every step copies its operands host->device, merges, and copies its
    # result (full capacity; the count comes back with it) device->host.
    # Three streams with their own buffers: a stream's next upload waits behind
    # its own download, so with three the uploads of steps i+1 and i+2 queue
    # back to back while step i merges and downloads (PCIe is full duplex).
    hin = [t.cpu().pin_memory() for t in (ak, av, bk, bv)]
    need = L.sort_reduce_workspace(na, nb, MAX_KEY)

    class Lane:
        def __init__(self):
            self.stream = torch.cuda.Stream()
            self.din = [torch.empty_like(t, device=dev) for t in hin]
            self.ok = torch.empty(n, dtype=torch.int64, device=dev)
            self.ov = torch.empty(n, dtype=torch.float64, device=dev)
            self.cnt = torch.zeros(1, dtype=torch.int64, device=dev)
            self.ws = L.workspace(need, dev)
            self.hok = torch.empty(n, dtype=torch.int64, pin_memory=True)
            self.hov = torch.empty(n, dtype=torch.float64, pin_memory=True)
            self.hcnt = torch.zeros(1, dtype=torch.int64, pin_memory=True)

    lanes = [Lane() for _ in range(E2E_LANES)]

    def e2e_step(i):
        ln = lanes[i % len(lanes)]
        with torch.cuda.stream(ln.stream):
            for d, h in zip(ln.din, hin):
                d.copy_(h, non_blocking=True)
            L.sort_reduce(ln.din[0], ln.din[1], ln.din[2], ln.din[3], max_key=MAX_KEY, a_rekey=spec,
                          out_keys=ln.ok, out_vals=ln.ov, count=ln.cnt, ws=ln.ws, sync=False)
            ln.hcnt.copy_(ln.cnt, non_blocking=True)
            ln.hok.copy_(ln.ok, non_blocking=True)
            ln.hov.copy_(ln.ov, non_blocking=True)

    e2e_steps = max(6, min(args.steps, 12))
    for i in range(len(lanes)):
        e2e_step(i)
    torch.cuda.synchronize()
    barrier(world)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for ln in lanes:
        ln.stream.wait_event(f0)
    for i in range(e2e_steps):
        e2e_step(i)
    for ln in lanes:
        ev = torch.cuda.Event()
        ev.record(ln.stream)
        stream.wait_event(ev)
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1) / e2e_steps, world)
    e2e_value = job_throughput(n, world, e2e_ms)
    m = int(lanes[0].hcnt.item())
    # the end-to-end result equals the (oracle-checked) device-resident one
    if m != n_out or not (np.array_equal(lanes[0].hok[:m].numpy(), out_k[:m].cpu().numpy())
                          and np.array_equal(lanes[0].hov[:m].numpy(), out_v[:m].cpu().numpy())):
        raise RuntimeError("end-to-end merge result differs from the device-resident one")

    # the same copies without the merge: the PCIe floor of an e2e step
    def copy_step(i):
        ln = lanes[i % len(lanes)]
        with torch.cuda.stream(ln.stream):
            for d, h in zip(ln.din, hin):
                d.copy_(h, non_blocking=True)
            ln.hcnt.copy_(ln.cnt, non_blocking=True)
            ln.hok.copy_(ln.ok, non_blocking=True)
            ln.hov.copy_(ln.ov, non_blocking=True)

    for i in range(len(lanes)):
        copy_step(i)
    torch.cuda.synchronize()
    barrier(world)
    f0.record(stream)
    for ln in lanes:
        ln.stream.wait_event(f0)
    for i in range(e2e_steps):
        copy_step(i)
    for ln in lanes:
        ev = torch.cuda.Event()
        ev.record(ln.stream)
        stream.wait_event(ev)
    f1.record(stream)
    torch.cuda.synchronize()
    copy_ms = max_over_ranks(f0.elapsed_time(f1) / e2e_steps, world)
    del lanes
    torch.cuda.empty_cache()

    # ---- roofline of the dominant kernel (largest share of the step) -------
    # algorithmic bytes per launch: a digit pass reads and writes every
    # (u64, f64) pair once; the bucket kernel reads every pair and writes every
    # output pair once.  DRAM traffic per pair from the committed
    # ncu summary of the merge.
    peak, peak_kind = peaks()
    prof_file = "onesweep8_bucket_merge_512x4_2x64M"
    cands = {
        "sort_onesweep": ("one digit pass (7 then 8 bits) of the bucketed sort over 2^27 (u64,f64) pairs", 32.0 * n,
                          "traffic_bytes_per_pair"),
        "bucket_sort_collect": ("per-bucket shared-memory sort + duplicate fold of the 2^27 pairs",
                                16.0 * n + 16.0 * n_out, "bucket_traffic_bytes_per_pair"),
    }
    # every timed merge kernel's algorithmic bytes and fraction of the HBM peak
    per_launch_bytes = {"sort_hist": 8.0 * n, "sort_onesweep": 32.0 * n,
                        "bucket_sort_collect": 16.0 * n + 16.0 * n_out}
    for name, b in per_launch_bytes.items():
        kk = kernels[name]
        if kk["launches"]:
            avg = kk["ms_total"] / kk["launches"]
            kk["alg_bytes_per_launch"] = b
            kk["hbm_frac"] = b / (avg * 1e-3) / 1e9 / peak
    dom = max(cands, key=lambda k: kernels[k]["ms_total"])
    desc, alg_bytes, tkey = cands[dom]
    avg_ms = kernels[dom]["ms_total"] / max(kernels[dom]["launches"], 1)
    achieved = alg_bytes / (avg_ms * 1e-3) / 1e9
    tpp = profile_traffic(prof_file, tkey)
    roofline = {"bound": "hbm", "kernel": f"{dom} ({desc})",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms,
                "traffic": (tpp * n) if tpp else None}
    step_alg = 16.0 * n + 16.0 * n_out
    extra = {}
    if world == 1 and not args.no_extra:
        # the metric's other two parts, measured in the same run: the skewed
        # contraction (products/s) and the emulated FP64 dense contraction
        del ak, av, bk, bv, out_k, out_v, ws
        torch.cuda.empty_cache()
        sub = argparse.Namespace(**vars(args))
        sub.steps, sub.warmup, sub.no_scheme1 = min(args.steps, 5), 3, True
        for key, fn in (("skewed_contraction", measure_skewed), ("dense", measure_dense),
                        ("batched", measure_batched), ("contraction", measure_contraction)):
            # (the 0.1 ms contraction replay keeps the full step count)
            d = fn(argparse.Namespace(**{**vars(sub), "steps": args.steps}) if key == "contraction" else sub)
            torch.cuda.empty_cache()
            if d is not None:
                extra[key] = {k: v for k, v in d.items() if k not in ("metric", "n_gpus", "scaling", "vs_baseline", "data")}
    result = None
    if rank == 0:
        cpu = None
        if world == 1 and not args.no_cpu:
            t, kind = cpu_merge_sample(CPU_SAMPLE, seed=7)
            cpu = {"value": 2 * CPU_SAMPLE / t, "unit": "nnz/s", "cores": 1, "kind": kind,
                   "sample": "one sortMerge of 2 x 2^23 nnz (1/8 of the workload, same distributions), "
                             + ("reference re-key + reference MSD radix sort" if kind == "reference"
                                else "restated re-key + sort") + " + restated collect_duplicates, single thread"}
        result = {
            "metric": METRIC, "value": value, "unit": "nnz/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nnz_per_operand": NNZ, "l2": L2_NOTE},
            "implementation": IMPLEMENTATION, "output_nnz": n_out,
            "parallelism": f"replicas x{world}" if world > 1 else "1 GPU",
            "oracle_check": check,
            "e2e": {"value": e2e_value, "unit": "nnz/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": int(16 * n), "d2h_bytes_per_step": int(16 * n + 8),
                    "pipelining": f"{E2E_LANES} streams: the H2D of steps i+1, i+2 overlap step i's merge and D2H",
                    "copy_only_ms_per_step": copy_ms,
                    "copy_only_note": "the same H2D and D2H copies per step with no merge (PCIe floor of a step)"},
            "gpu_launches": launches,
            "step_alg_bytes": step_alg, "step_hbm_frac_alg": step_alg / (ms * 1e-3) / 1e9 / peak,
            "kernels": kernels,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": sampler.summary(),
        }
        result.update(extra)
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


# ---------------------------------------------------------------------------
# other workloads (--workload ...): one JSON line each, same contract keys
# ---------------------------------------------------------------------------
def _line(metric_unit, value, ms, args, world, config, extra):
    d = {"metric": METRIC, "value": value, "unit": metric_unit, "n_gpus": world, "steps": args.steps,
         "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True, "scaling": "weak",
         "vs_baseline": None, "dtype": "f64", "data": "synthetic", "config": config}
    d.update(extra)
    return d


def _events():
    import torch
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def contraction_inputs(seed=0):
    """c(i,l) = a(i,j,k) * b(k,l,j): order-3 SparseMIA, dims 100^3, 10^4 distinct
    coordinates each (uniform without replacement), values U[-1,1], seed 0."""
    rng = np.random.default_rng(seed)
    ak = rng.choice(10 ** 6, 10 ** 4, replace=False).astype(np.uint64)
    bk = rng.choice(10 ** 6, 10 ** 4, replace=False).astype(np.uint64)
    return ak, rng.uniform(-1, 1, 10 ** 4), bk, rng.uniform(-1, 1, 10 ** 4)


def measure_contraction(args):
    """Plain sparse contraction, MIA level: toStraightLattice(a) (sort), toLatticeSort(b)
    (re-key to {2,0,1} + sort), csc_no_accum, all through the C ABI."""
    import torch

    import libnt_b200 as L
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    ak, av, bk, bv = contraction_inputs()
    hk = [torch.from_numpy(x.view(np.int64) if x.dtype == np.uint64 else x).pin_memory() for x in (ak, av, bk, bv)]
    dk = [torch.empty_like(x, device=dev) for x in hk]
    dims = [100, 100, 100]
    spec_a = L.RekeySpec.make(dims, [0, 1, 2], [0, 1, 2])
    spec_b = L.RekeySpec.make(dims, [0, 1, 2], [2, 0, 1])
    sa, sb = [torch.empty_like(x) for x in dk[:2]], [torch.empty_like(x) for x in dk[2:]]
    ws = L.workspace(L.permute_sort_workspace(10 ** 4, 10 ** 6), dev)
    out_h = [torch.empty(10 ** 4, dtype=torch.int64, pin_memory=True), torch.empty(10 ** 4, dtype=torch.float64,
                                                                                    pin_memory=True)]

    def step(host_io):
        if host_io:
            for d_, h_ in zip(dk, hk):
                d_.copy_(h_, non_blocking=True)
        L.permute_sort(dk[0], dk[1], max_key=10 ** 6, rekey=spec_a, out_keys=sa[0], out_vals=sa[1], ws=ws)
        L.permute_sort(dk[2], dk[3], max_key=10 ** 6, rekey=spec_b, out_keys=sb[0], out_vals=sb[1], ws=ws)
        ck, cv, prods = L.lattice_mult(sa[0], sa[1], sb[0], sb[1], 100, 10 ** 4, 100, 1)
        if host_io:
            out_h[0][:ck.numel()].copy_(ck)
            out_h[1][:cv.numel()].copy_(cv)
        return prods, ck.numel()

    for _ in range(args.warmup):
        prods, nc = step(True)
    torch.cuda.synchronize()
    launches0 = L.launch_count()
    e0, e1 = _events()
    e0.record()
    for _ in range(args.steps):
        step(False)
    e1.record()
    torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    launches = L.launch_count() - launches0
    f0, f1 = _events()
    f0.record()
    for _ in range(args.steps):
        step(True)
    f1.record()
    torch.cuda.synchronize()
    e2e_eager_ms = max_over_ranks(f0.elapsed_time(f1) / args.steps, world)

    # The same step as one CUDA graph: C-ABI calls on buffers sized from the
    # warm-up (the product count and output capacity of a fixed-shape
    # contraction), no host synchronisation inside; e2e adds the host copies.
    import ctypes as C
    lib = L.lib()
    A = L.Lattice.of(sa[0], sa[1], 100, 10 ** 4, 1)
    B = L.Lattice.of(sb[0], sb[1], 10 ** 4, 100, 1)
    nb_ = C.c_size_t(0)
    L._check(lib.lnt_lattice_mult_plan_workspace(C.byref(A), C.byref(B), C.byref(nb_)), "plan_workspace")
    plan = L.workspace(nb_.value, dev)
    L._check(lib.lnt_lattice_mult_workspace(C.byref(A), C.byref(B), C.c_uint64(prods), C.byref(nb_)), "workspace")
    mws = L.workspace(nb_.value, dev)
    counts = torch.zeros(2, dtype=torch.int64, device=dev)
    cap = 100 * 100
    gk = torch.empty(cap, dtype=torch.int64, device=dev)
    gv = torch.empty(cap, dtype=torch.float64, device=dev)
    gn = torch.zeros(1, dtype=torch.int64, device=dev)
    hn = torch.zeros(1, dtype=torch.int64, pin_memory=True)

    def graph_step(host_io):
        st = C.c_void_p(torch.cuda.current_stream().cuda_stream)
        if host_io:
            for d_, h_ in zip(dk, hk):
                d_.copy_(h_, non_blocking=True)
        L.permute_sort(dk[0], dk[1], max_key=10 ** 6, rekey=spec_a, out_keys=sa[0], out_vals=sa[1], ws=ws)
        L.permute_sort(dk[2], dk[3], max_key=10 ** 6, rekey=spec_b, out_keys=sb[0], out_vals=sb[1], ws=ws)
        L._check(lib.lnt_lattice_mult_plan(C.byref(A), C.byref(B), C.c_void_p(plan.data_ptr()), plan.numel(),
                                           C.c_void_p(counts.data_ptr()), st), "plan")
        L._check(lib.lnt_lattice_mult(C.byref(A), C.byref(B), C.c_void_p(plan.data_ptr()), C.c_uint64(prods),
                                      C.c_void_p(mws.data_ptr()), mws.numel(), C.c_void_p(gk.data_ptr()),
                                      C.c_void_p(gv.data_ptr()), C.c_void_p(gn.data_ptr()), st), "mult")
        if host_io:
            out_h[0][:nc].copy_(gk[:nc], non_blocking=True)
            out_h[1][:nc].copy_(gv[:nc], non_blocking=True)
            hn.copy_(gn, non_blocking=True)

    graph_ms, e2e_graph_ms = {}, {}
    sampler = ClockSampler(torch.cuda.current_device())
    for host_io, res in ((False, graph_ms), (True, e2e_graph_ms)):
        graph_step(host_io)
        torch.cuda.synchronize()
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g):
            graph_step(host_io)
        for _ in range(args.warmup):
            g.replay()
        torch.cuda.synchronize()
        h0, h1 = _events()
        with sampler if not host_io else contextlib.nullcontext():
            h0.record()
            for _ in range(args.steps):
                g.replay()
            h1.record()
            torch.cuda.synchronize()
        res["ms"] = max_over_ranks(h0.elapsed_time(h1) / args.steps, world)
        del g
    assert int(gn.item()) == nc and L.device_status() == 0
    ck_e, _, _ = L.lattice_mult(sa[0], sa[1], sb[0], sb[1], 100, 10 ** 4, 100, 1)
    assert torch.equal(ck_e, gk[:nc])
    eager_ms = ms
    ms = graph_ms["ms"]
    e2e_ms = e2e_graph_ms["ms"]
    if rank != 0:
        return None
    cpu = None
    if not args.no_cpu:
        import oracle
        t0 = time.perf_counter()
        reps = 20
        for _ in range(reps):
            a = oracle.SparseMIA(dims, ak, av, sorted=False)
            b = oracle.SparseMIA(dims, bk, bv, sorted=False)
            if oracle.ref_available():
                ka, va = oracle.ref_radix_sort(a.keys, a.vals, 10 ** 6)
                kb, vb = oracle.ref_radix_sort(oracle.ref_rekey(b.keys, dims, [0, 1, 2], [2, 0, 1]), b.vals, 10 ** 6)
            else:
                ka, va = oracle.sort_pairs(a.keys, a.vals)
                kb, vb = oracle.sort_pairs(oracle.rekey(b.keys, dims, [0, 1, 2], [2, 0, 1]), b.vals)
            oracle.lattice_mult(ka, va, 100, 10 ** 4, 1, kb, vb, 100)
        t = (time.perf_counter() - t0) / reps
        cpu = {"value": prods / t, "unit": "products/s", "cores": 1,
               "kind": "reference" if oracle.ref_available() else "port",
               "sample": "the full workload, median-free mean of 20 runs: reference sorts + restated csc_no_accum"}
    config = {"workload": "plain sparse contraction c(i,l)=a(i,j,k)*b(k,l,j), dims 100^3, 10^4 nnz each, "
                          "seed 0, both unsorted (sort a, re-key+sort b, csc_no_accum); a step = one CUDA-graph "
                          "replay of that sequence of C-ABI calls",
              "products": prods, "output_nnz": nc, "l2": "inputs fit in L2 (latency-bound workload)",
              "eager_ms_per_step": eager_ms, "eager_e2e_ms_per_step": e2e_eager_ms}
    return _line("products/s", prods * world / (ms * 1e-3), ms, args, world, config, {
        "e2e": {"value": prods * world / (e2e_ms * 1e-3), "unit": "products/s", "ms_per_step": e2e_ms,
                "h2d_bytes_per_step": 4 * 8 * 10 ** 4, "d2h_bytes_per_step": 16 * nc + 16},
        "gpu_launches": launches, "cpu_baseline": cpu, "clocks": sampler.summary(),
        "roofline": {"bound": "latency", "note": "about 0.5 MB of data: the step is launch- and latency-bound"},
    })


def run_contraction(args):
    d = measure_contraction(args)
    if d is not None:
        print(json.dumps(d), flush=True)
    return 0


def batched_inputs(count=4096, seed=0):
    """4096 problems c(i,l) = a(i,j,k) * b(k,l,j): dims U{16..512}, nnz per operand
    log-uniform in [1e2, 1e5] clamped to the tensor size, values U[-1,1].  Both
    operands are unsorted sets with keys in each tensor's own mode order (a: i
    fastest, then j, k; b: k fastest, then l, j).  Returns the lattice dims
    (h = di, w = dj dk, wB = dl, d = 1), the tensors' dims, the offsets, keys and
    values."""
    dims, tdims, ak, av, bk, bv = [], [], [], [], [], []
    for p in range(count):
        prng = np.random.default_rng([seed, p])
        i, j, k, l = (int(x) for x in prng.integers(16, 513, 4))
        na = min(int(round(10 ** prng.uniform(2, 5))), i * j * k)
        nb = min(int(round(10 ** prng.uniform(2, 5))), k * l * j)
        a = np.unique(prng.integers(0, i * j * k, int(na * 1.1) + 8, dtype=np.uint64))[:na]
        b = np.unique(prng.integers(0, k * l * j, int(nb * 1.1) + 8, dtype=np.uint64))[:nb]
        dims.append((i, j * k, l, 1))
        tdims.append(((i, j, k), (k, l, j)))
        ak.append(prng.permutation(a))
        bk.append(prng.permutation(b))
        av.append(prng.uniform(-1, 1, ak[-1].size))
        bv.append(prng.uniform(-1, 1, bk[-1].size))
    a_off = np.concatenate([[0], np.cumsum([x.size for x in ak])]).astype(np.uint64)
    b_off = np.concatenate([[0], np.cumsum([x.size for x in bk])]).astype(np.uint64)
    return np.array(dims, np.int64), tdims, a_off, b_off, ak, av, bk, bv


def batched_b_rows(bkeys, bdims):
    """Lattice rows (j + dj k) of b(k,l,j)'s keys (k fastest, then l, j)."""
    dk, dl, dj = bdims
    k = bkeys % dk
    j = bkeys // (dk * dl)
    return (j + dj * k).astype(np.int64)


def batched_expected(p, dims, tdims, ak, av, bk, bv, with_abs=False):
    """Problem p on the host: A sorted as it is, B re-keyed to {2,0,1} and sorted
    (the reference's toLatticeSort), then the restated csc_no_accum."""
    import oracle
    h, w, wB, _ = (int(x) for x in dims[p])
    oa = np.argsort(ak[p], kind="stable")
    kb = oracle.rekey(bk[p], tdims[p][1], [0, 1, 2], [2, 0, 1])
    ob = np.argsort(kb, kind="stable")
    return oracle.lattice_mult(ak[p][oa], av[p][oa], h, w, 1, kb[ob], bv[p][ob], wB, with_abs=with_abs)


def measure_batched(args):
    import torch

    import libnt_b200 as L
    import oracle
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    dims, tdims, a_off, b_off, ak, av, bk, bv = batched_inputs(count=args.batch_count, seed=rank)
    count = len(dims)
    cat = [np.concatenate(x) for x in (ak, av, bk, bv)]
    dt = [torch.from_numpy(x.view(np.int64) if x.dtype == np.uint64 else x).to(dev) for x in cat]
    b_specs = [L.RekeySpec.make(tdims[p][1], [0, 1, 2], [2, 0, 1]) for p in range(count)]
    batch = L.Batch(dims, a_off, b_off, *dt, a_rekey=[None] * count, b_rekey=b_specs)
    s = torch.cuda.Stream()
    s.wait_stream(torch.cuda.current_stream())
    with torch.cuda.stream(s):
        for _ in range(args.warmup):
            batch.run()
    torch.cuda.current_stream().wait_stream(s)
    torch.cuda.synchronize()
    # per-kernel device times of one eager run (the sort's roofline)
    L.profile_reset()
    L.profile_enable(True)
    batch.run()
    torch.cuda.synchronize()
    L.profile_enable(False)
    kernels = {}
    for name in ("batch_compose", "sort_hist", "sort_onesweep", "batch_colptr", "batch_spa_symbolic", "batch_scan",
                 "batch_spa_numeric", "batch_coff"):
        t, c = L.profile_query(name)
        kernels[name] = {"ms_total": t, "launches": c}
    L.profile_reset()
    g = torch.cuda.CUDAGraph()
    c0 = L.launch_count()
    with torch.cuda.graph(g):
        batch.run()
    per_replay = L.launch_count() - c0  # kernels recorded into the graph (a replay does not pass the host counter)
    for _ in range(args.warmup):
        g.replay()
    torch.cuda.synchronize()
    e0, e1 = _events()
    sampler = ClockSampler(torch.cuda.current_device())
    with sampler:
        e0.record()
        for _ in range(args.steps):
            g.replay()
        e1.record()
        torch.cuda.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    launches = per_replay * args.steps
    assert L.device_status() == 0, "device-side wait expired"
    out_total = int(batch.c_off[-1].item())
    # products per problem: over B entries, the size of the A column they meet
    products = 0
    for p in range(count):
        h, w = int(dims[p][0]), int(dims[p][1])
        cnt = np.bincount((ak[p] // h).astype(np.int64), minlength=w)
        products += int(cnt[batched_b_rows(bk[p], tdims[p][1])].sum())
    # oracle check on a sample of problems (the run fails on a mismatch)
    rng = np.random.default_rng(7)
    checked = 0
    for p in sorted(rng.choice(count, 64, replace=False).tolist()):
        ek, ev, ea = batched_expected(p, dims, tdims, ak, av, bk, bv, with_abs=True)
        k, v = batch.result(p)
        gk, gv = k.cpu().numpy().view(np.uint64), v.cpu().numpy()
        if not np.array_equal(gk, ek) or not np.all(np.abs(gv - ev) <= 1e-12 * ea):
            raise RuntimeError(f"batched problem {p} differs from the oracle")
        checked += 1
    # per-contraction loop on the same device, every problem: sort A, re-key and
    # sort B, plan + count read-back + product (C-ABI calls)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    lp = 0
    for p in range(0 if args.no_loop else count):
        a0, a1, b0, b1 = int(a_off[p]), int(a_off[p + 1]), int(b_off[p]), int(b_off[p + 1])
        h, w, wB, _ = (int(x) for x in dims[p])
        ka, va = L.permute_sort(dt[0][a0:a1], dt[1][a0:a1], max_key=h * w)
        kb, vb = L.permute_sort(dt[2][b0:b1], dt[3][b0:b1], max_key=w * wB, rekey=b_specs[p])
        _, _, pr = L.lattice_mult(ka, va, kb, vb, h, w, wB, 1)
        lp += pr
    torch.cuda.synchronize()
    loop_s = time.perf_counter() - t0
    if rank != 0:
        return None
    cpu = None
    if not args.no_cpu:
        n_cpu = 256
        kind = "reference" if oracle.ref_available() else "port"
        t0 = time.perf_counter()
        cp = 0
        for p in range(n_cpu):
            h, w, wB, _ = (int(x) for x in dims[p])
            if kind == "reference":
                ka, va = oracle.ref_radix_sort(ak[p], av[p], h * w)
                kb, vb = oracle.ref_radix_sort(oracle.ref_rekey(bk[p], tdims[p][1], [0, 1, 2], [2, 0, 1]), bv[p],
                                               w * wB)
            else:
                ka, va = oracle.sort_pairs(ak[p], av[p])
                kb, vb = oracle.sort_pairs(oracle.rekey(bk[p], tdims[p][1], [0, 1, 2], [2, 0, 1]), bv[p])
            oracle.lattice_mult(ka, va, h, w, 1, kb, vb, wB)
            cnt = np.bincount((ak[p] // h).astype(np.int64), minlength=w)
            cp += int(cnt[batched_b_rows(bk[p], tdims[p][1])].sum())
        t = time.perf_counter() - t0
        cpu = {"value": cp / t, "unit": "products/s", "cores": 1, "kind": kind,
               "sample": f"first {n_cpu} of the {count} problems from the same unsorted tensors: "
                         + ("the reference's radix sort of a, its re-key and radix sort of b"
                            if kind == "reference" else "restated sorts")
                         + ", restated csc_no_accum, one thread"}
    n_pairs = int(a_off[-1] + b_off[-1])
    os_ms, os_n = kernels["sort_onesweep"]["ms_total"], kernels["sort_onesweep"]["launches"]
    peak, peak_kind = peaks()
    avg = os_ms / max(os_n, 1)
    achieved = 32.0 * n_pairs / (avg * 1e-3) / 1e9 if os_n else 0.0
    config = {"workload": f"{count} independent sparse contractions c(i,l)=a(i,j,k)*b(k,l,j): dims U{{16..512}}, nnz "
                          "log-U[1e2,1e5] per operand, f64 U[-1,1], both operands unsorted tensors; a step = one "
                          "CUDA-graph replay of lnt_batched_contract (re-key, one segmented radix sort of all "
                          "operands, persistent SPA products)",
              "problems": count, "pairs_sorted": n_pairs, "products": products, "output_nnz": out_total,
              "queue_chunk": os.environ.get("LNT_BATCH_CHUNK") or tuned_value("batch_chunk"),
              "l2": "operands (1.9 GB) larger than the 126 MB L2"}
    return _line("products/s", products * world / (ms * 1e-3), ms, args, world, config, {
        "per_contraction_loop": None if args.no_loop else {
            "problems": count, "ms": loop_s * 1e3, "products_per_s": lp / loop_s,
            "note": "per problem: lnt_permute_sort of a, of b with its re-key, "
                    "lnt_lattice_mult_plan + count read-back + lnt_lattice_mult"},
        "oracle_check": {"problems": checked, "ok": True},
        "kernels": kernels,
        "gpu_launches": launches, "cpu_baseline": cpu, "clocks": sampler.summary(),
        "roofline": {"bound": "hbm", "kernel": f"sort_onesweep (one digit pass over the {n_pairs} composite-key pairs)",
                     "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                     "peak_source": peak_kind, "alg_bytes_per_launch": 32.0 * n_pairs, "avg_launch_ms": avg,
                     "traffic": None},
    })


def run_batched(args):
    d = measure_batched(args)
    if d is not None:
        print(json.dumps(d), flush=True)
    return 0


def run_dense(args):
    d = measure_dense(args)
    if d is not None:
        print(json.dumps(d), flush=True)
    return 0


def measure_dense(args):
    """c(i,j,m,n) = a(i,j,k,l) * b(k,l,m,n), all dims 128: a 16384^3 FP64 GEMM.
    Headline: scheme II (moduli + Chinese remaindering) on INT8 tensor cores;
    also timed: scheme I (INT8 slices) and the plain FP64 GEMM.  Returns the
    JSON line (rank 0) or None."""
    import torch

    import libnt_b200 as L
    import oracle
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    n = 1 << args.dense_log2
    g = torch.Generator(device=dev)
    g.manual_seed(5 + rank)
    results = {}
    flops = 2.0 * n ** 3
    reps = max(1, min(args.steps, 5))

    def timed(fn):
        for _ in range(max(1, args.warmup // 3)):
            fn()
        torch.cuda.synchronize()
        e0, e1 = _events()
        e0.record()
        for _ in range(reps):
            fn()
        e1.record()
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / reps

    rows = np.random.default_rng(1).integers(0, n, 1024)
    cols = np.random.default_rng(2).integers(0, n, 1024)
    idx = rows + n * cols
    for variant in ("uniform", "wide_exponent"):
        moduli = args.moduli if variant == "uniform" else max(args.moduli, 16)
        slices = args.slices if variant == "uniform" else max(args.slices, 8)
        if variant == "uniform":
            A = torch.rand(n * n, generator=g, device=dev, dtype=torch.float64) * 2 - 1
            B = torch.rand(n * n, generator=g, device=dev, dtype=torch.float64) * 2 - 1
        else:
            def wide():
                m = torch.rand(n * n, generator=g, device=dev, dtype=torch.float64) + 1
                e = torch.randint(-20, 21, (n * n,), generator=g, device=dev).to(torch.float64)
                sgn = torch.randint(0, 2, (n * n,), generator=g, device=dev).to(torch.float64) * 2 - 1
                return m * torch.pow(2.0, e) * sgn
            A, B = wide(), wide()
        Cc = torch.empty(n * n, dtype=torch.float64, device=dev)
        C64 = torch.empty(n * n, dtype=torch.float64, device=dev)
        ws64 = L.workspace(64 << 20, dev)
        t64 = timed(lambda: L.dense_mult_fp64(A, B, n, n, n, 1, out=C64, ws=ws64))
        wsc = L.workspace(L.dense_crt_workspace(n, n, n, moduli), dev)
        L.profile_reset()
        L.profile_enable(True)
        sampler = ClockSampler(torch.cuda.current_device())
        c0 = L.launch_count()
        with sampler:
            t_crt = timed(lambda: L.dense_mult_crt(A, B, n, n, n, 1, moduli, out=Cc, ws=wsc))
        per_call = (L.launch_count() - c0) // (reps + max(1, args.warmup // 3))
        L.profile_enable(False)
        kern = {k: L.profile_query(k)[0] / (reps + max(1, args.warmup // 3))
                for k in ("dense_residues", "dense_exp_a", "dense_exp_b", "dense_residue_a", "dense_residue_b",
                          "dense_mod_gemm", "dense_crt")}
        L.profile_reset()
        e2e = None
        if variant == "uniform" and not args.no_e2e:
            # the public call on operands copied from pinned host memory every
            # step, the product copied back; two streams with their own device
            # buffers, so that one step's uploads overlap the other's product
            # and download (as the merge's end-to-end line does)
            hA, hB = A.cpu().pin_memory(), B.cpu().pin_memory()

            class Lane:
                def __init__(self, C, ws):
                    self.stream = torch.cuda.Stream()
                    self.dA, self.dB = torch.empty_like(A), torch.empty_like(B)
                    self.C, self.ws = C, ws
                    self.hC = torch.empty(n * n, dtype=torch.float64, pin_memory=True)

            lanes = [Lane(Cc, wsc), Lane(torch.empty_like(Cc), L.workspace(L.dense_crt_workspace(n, n, n, moduli), dev))]

            def e2e_step(i):
                ln = lanes[i % len(lanes)]
                with torch.cuda.stream(ln.stream):
                    ln.dA.copy_(hA, non_blocking=True)
                    ln.dB.copy_(hB, non_blocking=True)
                    L.dense_mult_crt(ln.dA, ln.dB, n, n, n, 1, moduli, out=ln.C, ws=ln.ws)
                    ln.hC.copy_(ln.C, non_blocking=True)

            for i in range(len(lanes)):
                e2e_step(i)
            torch.cuda.synchronize()
            steps_e2e = max(4, reps)
            f0, f1 = _events()
            main = torch.cuda.current_stream()
            f0.record(main)
            for ln in lanes:
                ln.stream.wait_event(f0)
            for i in range(steps_e2e):
                e2e_step(i)
            for ln in lanes:
                ev = torch.cuda.Event()
                ev.record(ln.stream)
                main.wait_event(ev)
            f1.record(main)
            torch.cuda.synchronize()
            t_e2e = f0.elapsed_time(f1) / steps_e2e
            if not all(torch.equal(ln.hC, Cc.cpu()) for ln in lanes):
                raise RuntimeError("dense end-to-end product differs from the device-resident one")
            e2e = {"value": flops / (t_e2e * 1e-3) / 1e12, "unit": "TFLOP/s (FP64-equivalent)", "ms_per_step": t_e2e,
                   "h2d_bytes_per_step": 2 * 8 * n * n, "d2h_bytes_per_step": 8 * n * n,
                   "note": "lnt_dense_lattice_mult_crt on A and B copied from pinned host memory every step, "
                           "C copied back; two streams, each with its own buffers"}
            del lanes, hA, hB
        del wsc
        torch.cuda.empty_cache()
        Ah, Bh = A.cpu().numpy(), B.cpu().numpy()
        ref, mag = oracle.dense_entries(Ah, Bh, n, n, rows, cols)

        def errors(Cd):
            Ch = Cd.cpu().numpy()[idx]
            return (float(np.max(np.abs(Ch - ref) / mag)),
                    float(np.max(np.abs(Ch - ref) / np.maximum(np.abs(ref), 1e-300))),
                    float(np.max(np.abs(Ch - ref)) / np.max(np.abs(ref))))
        e_crt = errors(Cc)
        e_64 = errors(C64)
        full = float((Cc - C64).abs().max().item() / C64.abs().max().item())
        res = {"moduli": moduli, "crt_ms": t_crt, "fp64_ms": t64, "speedup_vs_fp64": t64 / t_crt,
               "effective_fp64_tflops": flops / (t_crt * 1e-3) / 1e12, "fp64_tflops": flops / (t64 * 1e-3) / 1e12,
               "max_err_rel_absAabsB": e_crt[0], "max_err_rel_C": e_crt[1], "max_err_over_max_C": e_crt[2],
               "fp64_gemm_err_rel_absAabsB": e_64[0], "fp64_gemm_err_rel_C": e_64[1],
               "max_diff_vs_fp64_over_maxC": full, "sampled_entries": int(rows.size),
               "kernels_ms_per_step": kern,
               "int8_tensor_tops": moduli * 2.0 * n ** 3 / (kern["dense_mod_gemm"] * 1e-3) / 1e12,
               "clocks": sampler.summary(), "e2e": e2e, "gpu_launches": per_call * reps}
        if not args.no_scheme1:
            wss = L.workspace(L.dense_split_workspace(n, n, n, slices), dev)
            t_split = timed(lambda: L.dense_mult_split(A, B, n, n, n, 1, slices, out=Cc, ws=wss))
            es = errors(Cc)
            res["scheme1_slices"] = {"slices": slices, "ms": t_split, "speedup_vs_fp64": t64 / t_split,
                                     "max_err_rel_absAabsB": es[0]}
            del wss
        results[variant] = res
        del A, B, Cc, C64
        torch.cuda.empty_cache()
    if rank != 0:
        return None
    # INT8 tensor peak measured here (torch._int_mm 8192^3), the roofline denominator
    a8 = torch.randint(-64, 64, (8192, 8192), device=dev, dtype=torch.int8)
    b8 = torch.randint(-64, 64, (8192, 8192), device=dev, dtype=torch.int8)
    for _ in range(3):
        torch._int_mm(a8, b8)
    torch.cuda.synchronize()
    e0, e1 = _events()
    e0.record()
    for _ in range(10):
        torch._int_mm(a8, b8)
    e1.record()
    torch.cuda.synchronize()
    int8_peak = 2 * 8192 ** 3 / (e0.elapsed_time(e1) / 10 * 1e-3) / 1e12
    cpu = None
    if not args.no_cpu:
        # the reference's GEMM is Eigen 3.2.5, which is not in the image: numpy's
        # float64 matmul on the host's BLAS stands in, on a bounded sample
        m = 4096
        hr = np.random.default_rng(3)
        Ah = hr.uniform(-1, 1, (m, m))
        Bh = hr.uniform(-1, 1, (m, m))
        Ah @ Bh
        best = float("inf")
        for _ in range(3):
            t0 = time.perf_counter()
            Ah @ Bh
            best = min(best, time.perf_counter() - t0)
        threads, blas = os.cpu_count(), "BLAS"
        try:
            from threadpoolctl import threadpool_info
            info = [i for i in threadpool_info() if i.get("user_api") == "blas"]
            if info:
                threads, blas = int(info[0].get("num_threads", threads)), str(info[0].get("internal_api", "BLAS"))
        except Exception:
            pass
        cpu = {"value": 2.0 * m ** 3 / best / 1e12, "unit": "TFLOP/s", "cores": threads, "kind": "port",
               "sample": f"numpy float64 matmul {m}^3 on the host's {blas} ({threads} threads), a labelled stand-in "
                         "for the reference's Eigen GEMM (not in the image); best of 3"}
    u = results["uniform"]
    config = {"workload": f"dense contraction c(i,j,m,n)=a(i,j,k,l)*b(k,l,m,n), dims 128 (a {n}^3 FP64 GEMM); "
                          "Ozaki scheme II: beta-bit integer operands, 13 (U[-1,1]) / 16 (2^+-20 exponents) moduli "
                          "<= 256 as INT8 tensor-core GEMMs (this library's tcgen05 kernel, products reduced "
                          "modulo m in its epilogue), Chinese remaindering in exact integer limbs",
              "variants": results}
    return _line("TFLOP/s (FP64-equivalent)", u["effective_fp64_tflops"], u["crt_ms"], args, world,
                 config, {
        "roofline": {"bound": "tensor", "kernel": "mod_gemm_kernel (tcgen05 INT8 products of all moduli, "
                                                  "reduced modulo m in the epilogue)", "achieved": u["int8_tensor_tops"],
                     "peak": int8_peak, "unit": "TOP/s", "frac": u["int8_tensor_tops"] / int8_peak,
                     "peak_source": "int8 torch._int_mm 8192^3 measured in this run (MEASURED_PEAKS.json has bf16 only)"},
        "vs_fp64_gemm": u["speedup_vs_fp64"], "clocks": u["clocks"], "cpu_baseline": cpu, "e2e": u["e2e"],
        "gpu_launches": u["gpu_launches"],
    })

def _timed_steps(torch, step, args):
    """W untimed steps, then K timed steps with CUDA events on the current
    stream (library profiler on); returns ms per step and the launch count."""
    import libnt_b200 as L
    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    launches0 = L.launch_count()
    L.profile_reset()
    L.profile_enable(True)
    sampler = ClockSampler(torch.cuda.current_device())
    e0, e1 = _events()
    with sampler:
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    L.profile_enable(False)
    return e0.elapsed_time(e1) / args.steps, L.launch_count() - launches0, sampler.summary()


def run_outer(args):
    """Product without contracted indices (noLatticeMult): d(i,l,!n) = a(i,!n) * b(!n,l),
    a 4096 x 65536 with 2^24 entries, b 65536 x 64 with 2^21 entries (uniform,
    distinct, key-sorted under [outer, inter]); a step = count + expansion
    through the C ABI.  Output-write bound: 16 B per product."""
    import ctypes as C

    import torch

    import libnt_b200 as L
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    h, wB, d = 4096 >> args.shrink, 64, 65536
    ak = torch.unique(torch.randint(0, h * d, (1 << (24 - args.shrink),), generator=g, device=dev))
    bk = torch.unique(torch.randint(0, wB * d, (1 << 21,), generator=g, device=dev))
    av = torch.rand(ak.numel(), generator=g, device=dev, dtype=torch.float64) * 2 - 1
    bv = torch.rand(bk.numel(), generator=g, device=dev, dtype=torch.float64) * 2 - 1
    A = L.Lattice.of(ak, av, h, 1, d)
    B = L.Lattice.of(bk, bv, 1, wB, d)
    lib = L.lib()
    nb_ = C.c_size_t(0)
    L._check(lib.lnt_nolattice_mult_workspace(C.byref(A), C.byref(B), C.byref(nb_)), "workspace")
    ws = L.workspace(nb_.value, dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)
    L._check(lib.lnt_nolattice_mult_count(C.byref(A), C.byref(B), C.c_void_p(ws.data_ptr()), ws.numel(),
                                          C.c_void_p(cnt.data_ptr()), stream), "count")
    P = int(cnt.item())
    ck = torch.empty(P, dtype=torch.int64, device=dev)
    cv = torch.empty(P, dtype=torch.float64, device=dev)

    def step():
        L._check(lib.lnt_nolattice_mult_count(C.byref(A), C.byref(B), C.c_void_p(ws.data_ptr()), ws.numel(),
                                              C.c_void_p(cnt.data_ptr()), stream), "count")
        L._check(lib.lnt_nolattice_mult(C.byref(A), C.byref(B), C.c_uint64(P), C.c_void_p(ws.data_ptr()),
                                        ws.numel(), C.c_void_p(ck.data_ptr()), C.c_void_p(cv.data_ptr()), stream),
                 "mult")

    ms, launches, clocks = _timed_steps(torch, step, args)
    exp_ms = L.profile_query("nolattice_expand")[0] / args.steps
    ms = max_over_ranks(ms, world)
    # spot check: the first and last products against the inputs
    k0 = int(ck[0].item())
    assert L.device_status() == 0 and int(cnt.item()) == P and bool(torch.all(ck[1:] >= ck[:-1]).item())
    if rank != 0:
        return 0
    peak, peak_kind = peaks()
    alg = 16.0 * (ak.numel() + bk.numel() + P)
    cpu = None
    if not args.no_cpu and world == 1:
        import oracle
        rng = np.random.default_rng(1)
        hs, ds = 512, 4096
        cak = np.unique(rng.integers(0, hs * ds, 1 << 20, dtype=np.uint64))
        cbk = np.unique(rng.integers(0, wB * ds, 1 << 17, dtype=np.uint64))
        t0 = time.perf_counter()
        kk, _ = oracle.nolattice_mult(cak, rng.uniform(-1, 1, cak.size), hs, ds, cbk, rng.uniform(-1, 1, cbk.size), wB)
        t = time.perf_counter() - t0
        cpu = {"value": kk.size / t, "unit": "products/s", "cores": 1, "kind": "port",
               "sample": f"a 512 x 4096 with 2^20 draws, b 64 x 4096 with 2^17 ({kk.size} products): the restated "
                         "noLatticeMult loop (numpy per inter index), one thread"}
    config = {"workload": "noLatticeMult d(i,l,!n) = a(i,!n) * b(!n,l): a 4096 x 65536 (2^24 draws), b 65536 x 64 "
                          "(2^21 draws), uniform, key-sorted; step = count + expansion",
              "nnz_a": int(ak.numel()), "nnz_b": int(bk.numel()), "products": P, "first_key": k0,
              "l2": "output far larger than L2", "parallelism": "1 GPU"}
    print(json.dumps(_line("products/s", P * world / (ms * 1e-3), ms, args, world, config, {
        "gpu_launches": launches, "cpu_baseline": cpu, "clocks": clocks,
        "roofline": {"bound": "hbm", "kernel": "nolattice_expand", "achieved": alg / (exp_ms * 1e-3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": alg / (exp_ms * 1e-3) / 1e9 / peak,
                     "alg_bytes_per_launch": alg, "avg_launch_ms": exp_ms, "peak_source": peak_kind,
                     "traffic": None},
    })), flush=True)
    return 0


def run_mixed(args):
    """Mixed lattice products: c(i,l) = A(i,j) * s(j,l) with A dense 2048 x 8192
    (128 MB, about the L2) and s sparse 8192 x 16384 with 2^21 distinct uniform
    entries (128 per column), key-sorted column-major; a step = count +
    product through the C ABI (dense x sparse).  The sparse x dense product
    s'(l,j) * A'(j,i) on the transposed data (its transpose of the dense operand
    included) is timed the same way and reported in config.  Each (entry, row)
    is one multiply and one add on an element of A gathered from L2."""
    import ctypes as C

    import torch

    import libnt_b200 as L
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    h, w, wB = 2048, 8192, 16384 >> args.shrink
    nnz = 1 << (21 - args.shrink)
    A = torch.rand(h * w, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    sk = torch.unique(torch.randint(0, w * wB, (nnz,), generator=g, device=dev))
    sv = torch.rand(sk.numel(), generator=g, device=dev, dtype=torch.float64) * 2 - 1
    lib = L.lib()
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def setup(D, S, other, dense_first):
        nb_ = C.c_size_t(0)
        L._check(lib.lnt_sparse_dense_mult_workspace(C.byref(S), other, dense_first, C.byref(nb_)), "workspace")
        ws = L.workspace(nb_.value, dev)
        cnt = torch.zeros(1, dtype=torch.int64, device=dev)
        L._check(lib.lnt_sparse_dense_mult_count(C.byref(S), other, dense_first, C.c_void_p(ws.data_ptr()),
                                                 ws.numel(), C.c_void_p(cnt.data_ptr()), stream), "count")
        n_out = int(cnt.item())
        ck = torch.empty(n_out, dtype=torch.int64, device=dev)
        cv = torch.empty(n_out, dtype=torch.float64, device=dev)

        def step():
            L._check(lib.lnt_sparse_dense_mult_count(C.byref(S), other, dense_first, C.c_void_p(ws.data_ptr()),
                                                     ws.numel(), C.c_void_p(cnt.data_ptr()), stream), "count")
            L._check(lib.lnt_sparse_dense_mult(C.c_void_p(D.data_ptr()), C.byref(S), other, dense_first,
                                               C.c_void_p(ws.data_ptr()), ws.numel(), C.c_void_p(ck.data_ptr()),
                                               C.c_void_p(cv.data_ptr()), stream), "mult")
        return step, n_out, ck, cv

    S = L.Lattice.of(sk, sv, w, wB, 1)
    step, n_out, ck, cv = setup(A, S, h, 1)
    ms, launches, clocks = _timed_steps(torch, step, args)
    prod_ms = L.profile_query("mixed_product")[0] / args.steps
    ms = max_over_ranks(ms, world)
    # spot check: the first output against a float64 recomputation from the inputs
    col = int(ck[0].item()) // h
    rows = sk[(sk // w) == col] % w
    vals = sv[(sk // w) == col]
    acc = torch.zeros((), dtype=torch.float64, device=dev)
    for r, v in zip(rows.tolist(), vals.tolist()):
        acc = acc + v * A[int(r) * h]
    assert L.device_status() == 0 and n_out == int(torch.unique(sk // w).numel()) * h
    assert float(acc.item()) == float(cv[0].item())
    # sparse x dense on the transposed operands, c'(l,i) = s'(l,j) * B(j,i) with s' = s^T (its row-major
    # keys j + w l are s's column-major keys) and B = A^T (w x h, column-major)
    S2 = L.Lattice.of(sk, sv, wB, w, 1)
    step2, _, _, _ = setup(A.view(w, h).t().contiguous().view(-1), S2, h, 0)
    ms2, _, _ = _timed_steps(torch, step2, args)
    sd_kernels = {k: L.profile_query(k)[0] / args.steps for k in ("mixed_count", "mixed_transpose", "mixed_product")}
    if rank != 0:
        return 0
    peak, peak_kind = peaks()
    flops = 2.0 * sk.numel() * h
    alg = 8.0 * h * w + 16.0 * sk.numel() + 16.0 * n_out
    gathered = 8.0 * sk.numel() * h
    cpu = None
    if not args.no_cpu and world == 1:
        import oracle
        rng = np.random.default_rng(1)
        cw, cwB = 8192, 64
        cA = rng.uniform(-1, 1, h * cw)
        csk = np.unique(rng.integers(0, cw * cwB, 1 << 13, dtype=np.uint64))
        t0 = time.perf_counter()
        oracle.dense_sparse_mult(cA, csk, rng.uniform(-1, 1, csk.size), h, cw, cwB, 1)
        t = time.perf_counter() - t0
        cpu = {"value": 2.0 * csk.size * h / t / 1e9, "unit": "GFLOP/s", "cores": 1, "kind": "port",
               "sample": f"A 2048 x 8192, s 8192 x 64 with {csk.size} entries: the restated dense x sparse loop "
                         "(numpy, one column of A per entry), one thread"}
    config = {"workload": "dense x sparse c(i,l) = A(i,j) * s(j,l): A 2048 x 8192 dense, s 8192 x 16384 with "
                          "2^21 uniform distinct entries; step = count + product",
              "nnz": int(sk.numel()), "outputs": n_out, "product_ms": prod_ms,
              "l2_gather_GBs": gathered / (prod_ms * 1e-3) / 1e9,
              "sparse_x_dense_ms_per_step": ms2, "sparse_x_dense_kernels_ms": sd_kernels,
              "l2": "A (128 MB) about the L2; the output (537 MB) far larger", "parallelism": "1 GPU"}
    print(json.dumps(_line("GFLOP/s", flops * world / (ms * 1e-3) / 1e9, ms, args, world, config, {
        "gpu_launches": launches, "cpu_baseline": cpu, "clocks": clocks,
        "roofline": {"bound": "hbm", "kernel": "mixed_product", "achieved": alg / (prod_ms * 1e-3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": alg / (prod_ms * 1e-3) / 1e9 / peak,
                     "alg_bytes_per_launch": alg, "avg_launch_ms": prod_ms, "peak_source": peak_kind,
                     "traffic": None},
    })), flush=True)
    return 0


def run_unary(args):
    """Unary contraction (contract_attract): b(k) = a(i,i,k), a 8192 x 8192 x 1024
    with 2^26 entries (uniform, distinct, key-sorted under [i, i, k]); a step =
    lnt_contract_attract through the C ABI.  HBM bound: 16 B per input entry
    plus 16 B per output entry."""
    import torch

    import libnt_b200 as L
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    dims = [8192, 8192, 1024 >> args.shrink]
    total = dims[0] * dims[1] * dims[2]
    keys = torch.unique(torch.randint(0, total, (1 << (26 - args.shrink),), generator=g, device=dev))
    # a tenth of the entries on the diagonal i = i', so the output is not trivial
    idx = torch.arange(0, keys.numel(), 10, device=dev)
    i0 = keys[idx] % dims[0]
    rest = keys[idx] // (dims[0] * dims[1])
    keys[idx] = i0 + dims[0] * i0 + dims[0] * dims[1] * rest
    keys = torch.unique(keys)
    vals = torch.rand(keys.numel(), generator=g, device=dev, dtype=torch.float64) * 2 - 1
    n = keys.numel()
    import ctypes as C
    lib = L.lib()
    nb_ = C.c_size_t(0)
    L._check(lib.lnt_contract_attract_workspace(n, C.byref(nb_)), "workspace")
    ws = L.workspace(nb_.value, dev)
    ok = torch.empty(n, dtype=torch.int64, device=dev)
    ov = torch.empty(n, dtype=torch.float64, device=dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)
    sd = np.array(dims, np.int64)
    cp = np.array([2], np.int32)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def step():
        L._check(lib.lnt_contract_attract(C.c_void_p(keys.data_ptr()), C.c_void_p(vals.data_ptr()), n, 3,
                                          sd.ctypes.data, 1, cp.ctypes.data, 0, None, C.c_void_p(ok.data_ptr()),
                                          C.c_void_p(ov.data_ptr()), C.c_void_p(cnt.data_ptr()), None,
                                          C.c_void_p(ws.data_ptr()), ws.numel(), stream), "lnt_contract_attract")

    ms, launches, clocks = _timed_steps(torch, step, args)
    kernels = {k: L.profile_query(k)[0] / args.steps for k in ("unary_map", "collect_lead", "collect", "unary_scan",
                                                                 "unary_write")}
    ms = max_over_ranks(ms, world)
    m = int(cnt.item())
    # spot check: output k holds the sum of the diagonal entries a(i,i,k)
    kk = keys.cpu().numpy()
    diag = (kk % dims[0]) == ((kk // dims[0]) % dims[1])
    ref = np.bincount(kk[diag] // (dims[0] * dims[1]), weights=vals.cpu().numpy()[diag], minlength=dims[2])
    got = np.zeros(dims[2])
    got[ok[:m].cpu().numpy()] = ov[:m].cpu().numpy()
    assert L.device_status() == 0 and np.allclose(got, ref, rtol=0, atol=1e-9)
    if rank != 0:
        return 0
    peak, peak_kind = peaks()
    alg = 16.0 * (n + m)
    config = {"workload": "contract_attract b(k) = a(i,i,k): a 8192 x 8192 x 1024, 2^26 entries (a tenth on the "
                          "diagonal), uniform, key-sorted; step = lnt_contract_attract (map, fold, scan, write)",
              "nnz": int(n), "output_nnz": int(m), "l2": "input far larger than L2", "parallelism": "1 GPU"}
    print(json.dumps(_line("nnz/s", n * world / (ms * 1e-3), ms, args, world, config, {
        "gpu_launches": launches, "cpu_baseline": None, "clocks": clocks, "kernels_ms_per_step": kernels,
        "roofline": {"bound": "hbm", "kernel": "whole contract_attract call (4 kernels + the fold)",
                     "achieved": alg / (ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (ms * 1e-3) / 1e9 / peak, "alg_bytes_per_launch": alg, "avg_launch_ms": ms,
                     "peak_source": peak_kind, "traffic": None},
    })), flush=True)
    return 0


def run_scanmerge(args):
    """The merge workload with both operands already sorted (each under its
    default sequence): perform_outside_merge sorts A into B's order (sort(seq):
    re-key {0,1,2,3} -> {3,2,1,0} + sort) and merges linearly.  A step =
    lnt_permute_sort(A) + lnt_merge_sorted(A', B) through the C ABI."""
    import ctypes as C

    import torch

    import libnt_b200 as L
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    g = torch.Generator(device=dev)
    g.manual_seed(0)
    n = 1 << args.nnz_log2
    ak = torch.sort(torch.randint(0, MAX_KEY, (n,), generator=g, device=dev)).values
    bk = torch.sort(torch.randint(0, MAX_KEY, (n,), generator=g, device=dev)).values
    av = torch.rand(n, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    bv = torch.rand(n, generator=g, device=dev, dtype=torch.float64) * 2 - 1
    spec = L.RekeySpec.make(DIMS, [0, 1, 2, 3], [3, 2, 1, 0])
    sk, sv = torch.empty_like(ak), torch.empty_like(av)
    ws_s = L.workspace(L.permute_sort_workspace(n, MAX_KEY), dev)
    lib = L.lib()
    nb_ = C.c_size_t(0)
    L._check(lib.lnt_merge_sorted_workspace(n, n, C.byref(nb_)), "merge workspace")
    ws_m = L.workspace(nb_.value, dev)
    ok = torch.empty(2 * n, dtype=torch.int64, device=dev)
    ov = torch.empty(2 * n, dtype=torch.float64, device=dev)
    cnt = torch.zeros(1, dtype=torch.int64, device=dev)

    def step():
        L.permute_sort(ak, av, max_key=MAX_KEY, rekey=spec, out_keys=sk, out_vals=sv, ws=ws_s)
        L.merge_sorted(sk, sv, bk, bv, 0, out_keys=ok, out_vals=ov, count=cnt, ws=ws_m, sync=False)

    ms, launches, clocks = _timed_steps(torch, step, args)
    kernels = {k: L.profile_query(k)[0] / args.steps for k in ("sort_hist", "sort_onesweep", "merge")}
    ms = max_over_ranks(ms, world)
    m = int(cnt.item())
    assert L.device_status() == 0 and bool(torch.all(ok[1:m] >= ok[:m - 1]).item())  # duplicates within an operand stay
    if rank != 0:
        return 0
    peak, peak_kind = peaks()
    mg = kernels["merge"]
    alg = 32.0 * n + 16.0 * m
    config = {"workload": "sparse merge c(i,j,k,l)=a(i,j,k,l)+b(l,k,j,i), 512^4, 2^%d nnz per operand, both "
                          "operands sorted (outside_scanMerge: sort(seq) of a into b's order, linear merge)"
                          % args.nnz_log2, "output_nnz": m, "l2": "inputs larger than L2", "parallelism": "1 GPU"}
    print(json.dumps(_line("nnz/s", 2 * n * world / (ms * 1e-3), ms, args, world, config, {
        "gpu_launches": launches, "kernels_ms_per_step": kernels, "cpu_baseline": None, "clocks": clocks,
        "roofline": {"bound": "hbm", "kernel": "merge_kernel (the linear merge)", "achieved": alg / (mg * 1e-3) / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": alg / (mg * 1e-3) / 1e9 / peak,
                     "alg_bytes_per_launch": alg, "avg_launch_ms": mg, "peak_source": peak_kind, "traffic": None},
    })), flush=True)
    return 0


SKEW_DIMS = (1024, 1024, 256, 256, 4096)  # a(i,j,k,l), b(k,l,m)


def _zipf_cdf(dim, xp, **kw):
    p = xp.arange(1, dim + 1, **kw) ** -1.1
    return xp.cumsum(p / p.sum(), 0)


def skewed_inputs_gpu(dev, nnz_a, nnz_b, dims=SKEW_DIMS, seed=0):
    """c(i,j,m) = a(i,j,k,l) * b(k,l,m): (k,l) ~ Zipf(1.1) truncated to the mode
    extent, rank r -> coordinate r-1 in both operands (aligned), i, j, m uniform,
    values N(0,1), duplicate coordinates collapsed.  Returned as key-sorted
    lattices A (rows (i,j), cols (k,l)) and B (rows (k,l), cols m)."""
    import torch
    g = torch.Generator(device=dev)
    g.manual_seed(seed)
    di, dj, dk, dl, dm = dims

    def zipf(n, dim):
        cdf = _zipf_cdf(dim, torch, dtype=torch.float64, device=dev)
        u = torch.rand(n, generator=g, device=dev, dtype=torch.float64)
        return torch.searchsorted(cdf, u).clamp_(max=dim - 1)

    i = torch.randint(0, di, (nnz_a,), generator=g, device=dev)
    j = torch.randint(0, dj, (nnz_a,), generator=g, device=dev)
    ak = torch.unique((i + di * j) + (di * dj) * (zipf(nnz_a, dk) + dk * zipf(nnz_a, dl)))
    del i, j
    kb, lb = zipf(nnz_b, dk), zipf(nnz_b, dl)
    m = torch.randint(0, dm, (nnz_b,), generator=g, device=dev)
    bk = torch.unique((kb + dk * lb) + (dk * dl) * m)
    del kb, lb, m
    av = torch.randn(ak.numel(), generator=g, device=dev, dtype=torch.float64)
    bv = torch.randn(bk.numel(), generator=g, device=dev, dtype=torch.float64)
    return ak, av, bk, bv


def skewed_inputs_cpu(nnz_a, nnz_b, dims=SKEW_DIMS, seed=0):
    """The same distributions drawn with numpy (for the CPU baseline sample)."""
    rng = np.random.default_rng(seed)
    di, dj, dk, dl, dm = dims

    def zipf(n, dim):
        return np.minimum(np.searchsorted(_zipf_cdf(dim, np, dtype=np.float64), rng.random(n)), dim - 1)

    i, j = rng.integers(0, di, nnz_a), rng.integers(0, dj, nnz_a)
    ak = np.unique((i + di * j) + (di * dj) * (zipf(nnz_a, dk) + dk * zipf(nnz_a, dl))).astype(np.uint64)
    bk = np.unique((zipf(nnz_b, dk) + dk * zipf(nnz_b, dl)) + (dk * dl) * rng.integers(0, dm, nnz_b)).astype(
        np.uint64)
    return ak, rng.standard_normal(ak.size), bk, rng.standard_normal(bk.size)


def run_skewed(args):
    d = measure_skewed(args)
    if d is not None:
        print(json.dumps(d), flush=True)
    return 0


def measure_skewed(args):
    """Large skewed sparse contraction c(i,j,m) = a(i,j,k,l) * b(k,l,m) on
    key-sorted lattices; a step = lnt_lattice_mult_plan (product count) +
    lnt_lattice_mult (the tile engine at this shape) through the C ABI.
    Returns the JSON line (rank 0) or None."""
    import ctypes as C

    import torch

    import libnt_b200 as L
    world, rank, local = dist_setup(args.gpus)
    dev = torch.device("cuda", torch.cuda.current_device())
    dims = tuple(int(x) for x in args.skew_dims.split(","))
    di, dj, dk, dl, dm = dims
    h, w, wB = di * dj, dk * dl, dm
    nnz = 1 << args.skew_log2
    nnz_b = 1 << (args.skew_b_log2 if args.skew_b_log2 is not None else args.skew_log2)
    ak, av, bk, bv = skewed_inputs_gpu(dev, nnz, nnz_b, dims)
    A = L.Lattice.of(ak, av, h, w, 1)
    B = L.Lattice.of(bk, bv, w, wB, 1)
    lib = L.lib()
    nb_ = C.c_size_t(0)
    L._check(lib.lnt_lattice_mult_plan_workspace(C.byref(A), C.byref(B), C.byref(nb_)), "plan_workspace")
    plan = L.workspace(nb_.value, dev)
    counts = torch.zeros(2, dtype=torch.int64, device=dev)
    stream = C.c_void_p(torch.cuda.current_stream().cuda_stream)

    def run_plan():
        L._check(lib.lnt_lattice_mult_plan(C.byref(A), C.byref(B), C.c_void_p(plan.data_ptr()), plan.numel(),
                                           C.c_void_p(counts.data_ptr()), stream), "lnt_lattice_mult_plan")

    run_plan()
    products, cap = (int(x) for x in counts.tolist())
    L._check(lib.lnt_lattice_mult_workspace(C.byref(A), C.byref(B), C.c_uint64(products), C.byref(nb_)),
             "lnt_lattice_mult_workspace")
    ws = L.workspace(nb_.value, dev)
    ck = torch.empty(max(cap, 1), dtype=torch.int64, device=dev)
    cv = torch.empty(max(cap, 1), dtype=torch.float64, device=dev)
    nc = torch.zeros(1, dtype=torch.int64, device=dev)

    def step():
        run_plan()
        L._check(lib.lnt_lattice_mult(C.byref(A), C.byref(B), C.c_void_p(plan.data_ptr()), C.c_uint64(products),
                                      C.c_void_p(ws.data_ptr()), ws.numel(), C.c_void_p(ck.data_ptr()),
                                      C.c_void_p(cv.data_ptr()), C.c_void_p(nc.data_ptr()), stream),
                 "lnt_lattice_mult")

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    n_out = int(nc.item())
    assert L.device_status() == 0
    assert 0 < n_out <= cap, (n_out, cap)
    # spot check: 64 output entries (exact integer positions) against a float64 recomputation from the inputs
    sel = torch.from_numpy((np.arange(64, dtype=np.int64) * (n_out - 1)) // 63).to(dev)
    keys, vals = ck[sel].cpu().numpy(), cv[sel].cpu().numpy()
    akh, avh, bkh, bvh = (x.cpu().numpy() for x in (ak, av, bk, bv))
    a_col, a_row = akh // h, akh % h
    spot = 0.0
    for key, val in zip(keys, vals):
        r, col = int(key) % h, int(key) // h
        sa = a_row == r
        cs, va = a_col[sa], avh[sa]
        bpos = np.searchsorted(bkh, cs + w * col)
        hit = (bpos < bkh.size) & (bkh[np.minimum(bpos, bkh.size - 1)] == cs + w * col)
        terms = va[hit] * bvh[bpos[hit]]
        assert hit.any()
        spot = max(spot, abs(val - terms.sum()) / max(np.abs(terms).sum(), 1e-300))
    assert spot <= 1e-12, spot
    launches0 = L.launch_count()
    L.profile_reset()
    L.profile_enable(True)
    sampler = ClockSampler(torch.cuda.current_device())
    e0, e1 = _events()
    with sampler:
        torch.cuda.synchronize()
        barrier(world)
        e0.record()
        for _ in range(args.steps):
            step()
        e1.record()
        torch.cuda.synchronize()
    L.profile_enable(False)
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world)
    launches = L.launch_count() - launches0
    names = ("spgemm_colptr", "spgemm_count", "sort_hist", "sort_onesweep", "collect", "tile_rowptr", "tile_bprep",
             "tile_cbits", "tile_count", "tile_scan", "tile_numeric")
    kernels = {k: L.profile_query(k)[0] / args.steps for k in names}
    if rank != 0:
        return None
    peak, peak_kind = peaks()
    alg = 16.0 * (ak.numel() + bk.numel() + n_out)
    num_ms = kernels["tile_numeric"]
    tpo = profile_traffic("tile_numeric_skewed_2x32M", "traffic_bytes_per_output")
    cpu = None
    if not args.no_cpu and world == 1:
        import oracle
        sample_log2 = args.skew_cpu_log2
        cak, cav, cbk, cbv = skewed_inputs_cpu(1 << sample_log2, 1 << sample_log2, dims)
        t0 = time.perf_counter()
        ok, _ = oracle.lattice_mult(cak, cav, h, w, 1, cbk, cbv, wB)
        t = time.perf_counter() - t0
        a_cnt = np.bincount((cak // h).astype(np.int64), minlength=w)
        b_cnt = np.bincount((cbk % w).astype(np.int64), minlength=w)
        p_cpu = int((a_cnt * b_cnt).sum())
        cpu = {"value": p_cpu / t, "unit": "products/s", "cores": 1, "kind": "port",
               "sample": f"same dims and distributions at 2^{sample_log2} nnz per operand ({p_cpu:.3e} products, "
                         f"{ok.size} output nnz): restated csc_no_accum (per-column scatter, sort, fold), one thread; "
                         "products/s is normalised by that sample's product count"}
    config = {"workload": f"skewed sparse contraction c(i,j,m)=a(i,j,k,l)*b(k,l,m), a dims {di}x{dj}x{dk}x{dl}, "
                          f"b dims {dk}x{dl}x{dm}, {nnz} / {nnz_b} coordinates drawn for a / b "
                          "(duplicates collapsed), (k,l) Zipf(1.1) aligned, values N(0,1); step = plan + tile-engine "
                          "product on key-sorted lattices",
              "nnz_a": int(ak.numel()), "nnz_b": int(bk.numel()), "products": products, "output_nnz": n_out,
              "l2": "output (16 B x output nnz) far larger than L2", "parallelism": "1 GPU"}
    return _line("products/s", products * world / (ms * 1e-3), ms, args, world, config, {
        "gpu_launches": launches, "kernels_ms_per_step": kernels, "spot_check_max_rel_err": spot,
        "roofline": {"bound": "hbm", "kernel": "tile_numeric (products, staging, output write)",
                     "achieved": alg / (num_ms * 1e-3) / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": alg / (num_ms * 1e-3) / 1e9 / peak, "alg_bytes_per_launch": alg,
                     "avg_launch_ms": num_ms, "peak_source": peak_kind,
                     "step_frac": alg / (ms * 1e-3) / 1e9 / peak,
                     "traffic": (tpo * n_out) if tpo else None,
                     "traffic_note": "DRAM bytes per output entry from the small-case ncu capture, times the output count"},
        "cpu_baseline": cpu, "clocks": sampler.summary(),
    })


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu", action="store_true", help="skip the CPU baseline leg")
    ap.add_argument("--nnz-log2", type=int, default=26,
                    help="log2 of non-zeros per operand (26 = the workload; smaller only for profiling)")
    ap.add_argument("--no-e2e", action="store_true", help="device-resident timing only (profiling runs)")
    ap.add_argument("--no-extra", action="store_true",
                    help="merge line only: skip the skewed-contraction, dense, batched and contraction keys")
    ap.add_argument("--workload", default="merge", choices=["merge", "contraction", "batched", "dense", "skewed", "outer", "unary", "scanmerge", "mixed"],
                    help="merge (default: the sparse merge under permutation), contraction (100^3 plain "
                         "contraction), batched (4096 uneven contractions), dense (128^4 dense contraction)")
    ap.add_argument("--slices", type=int, default=7, help="dense scheme I: INT8 slices per operand")
    ap.add_argument("--moduli", type=int, default=13, help="dense scheme II: moduli (uniform data)")
    ap.add_argument("--no-scheme1", action="store_true", help="dense: skip timing scheme I")
    ap.add_argument("--dense-log2", type=int, default=14, help="dense: log2 of the GEMM size (14 = the workload)")
    ap.add_argument("--batch-count", type=int, default=4096, help="batched: problems (4096 = the workload)")
    ap.add_argument("--no-loop", action="store_true", help="batched: skip the per-contraction loop (profiling)")
    ap.add_argument("--skew-log2", type=int, default=25, help="skewed: log2 of coordinates drawn per operand")
    ap.add_argument("--shrink", type=int, default=0, help="outer / unary: divide the workload by 2^shrink (profiling)")
    ap.add_argument("--skew-b-log2", type=int, default=None, help="skewed: log2 of coordinates drawn for b "
                                                                   "(default: --skew-log2)")
    ap.add_argument("--skew-dims", default=",".join(map(str, SKEW_DIMS)),
                    help="skewed: i,j,k,l,m extents (default: the workload's)")
    ap.add_argument("--skew-cpu-log2", type=int, default=18, help="skewed: CPU baseline sample size (log2 nnz)")
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        if args.workload != "merge":
            print(json.dumps({"impl": "reference", "unavailable": "reference arm implemented for the merge workload"}))
            return 0
        return run_reference(args)
    return {"merge": run_ours, "contraction": run_contraction, "batched": run_batched,
            "dense": run_dense, "skewed": run_skewed, "outer": run_outer, "unary": run_unary,
            "scanmerge": run_scanmerge, "mixed": run_mixed}[args.workload](args)


if __name__ == "__main__":
    sys.exit(main())

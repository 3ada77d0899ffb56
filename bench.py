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
            "re-key A to {3,2,1,0}, concatenate, LSD radix sort of 2^27 (u64,f64) pairs, collect duplicates)")
HBM_FALLBACK_GBS = 6650.0


def peaks():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return HBM_FALLBACK_GBS, "fallback"


def profile_traffic(name: str):
    """Per-pair DRAM traffic of a kernel from the committed ncu summary
    (line 'traffic_bytes_per_pair: X'), or None."""
    f = ROOT / "profiles" / f"{name}.md"
    if not f.exists():
        return None
    for line in f.read_text().splitlines():
        if line.strip().startswith("traffic_bytes_per_pair:"):
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
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


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


def run_reference(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    times = []
    kind = "port"
    for i in range(args.warmup + args.steps):
        t, kind = cpu_merge_sample(CPU_SAMPLE, seed=i)
        if i >= args.warmup:
            times.append(t)
    t = statistics.median(times)
    rate = 2 * CPU_SAMPLE / t
    sample = (f"2 x 2^23 nnz per step (1/8 of the 2 x 2^26 workload, same distributions), "
              f"{'reference re-key + reference MSD radix sort' if kind == 'reference' else 'restated re-key + sort'}"
              f" + restated collect_duplicates, single thread")
    line = {"impl": "reference", "metric": METRIC, "value": rate, "unit": "nnz/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3 * (NNZ / CPU_SAMPLE),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": WORKLOAD, "nnz_per_operand": NNZ, "parallelism": "single host thread"},
            "cpu_baseline": {"value": rate, "unit": "nnz/s", "cores": 1, "kind": kind, "sample": sample},
            "e2e": {"value": rate, "unit": "nnz/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
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
    value = n * world / (ms * 1e-3)
    os_ms, os_launches = L.profile_query("sort_onesweep")
    kernels = {}
    for name in ("sort_hist", "sort_onesweep", "collect_lead", "collect"):
        t, c = L.profile_query(name)
        kernels[name] = {"ms_total": t, "launches": c}
    L.profile_reset()
    n_out = int(cnt.item())
    assert L.device_status() == 0, "device-side wait expired during timing"

    if args.no_e2e:
        if rank == 0:
            print(json.dumps({"metric": METRIC, "value": value, "unit": "nnz/s", "ms_per_step": ms,
                              "nnz_per_operand": na, "kernels": kernels}), flush=True)
        return 0

    # ---- end-to-end through the C ABI from pinned host buffers ------------
    hk_a = ak.cpu().pin_memory()
    hv_a = av.cpu().pin_memory()
    hk_b = bk.cpu().pin_memory()
    hv_b = bv.cpu().pin_memory()
    ho_k = torch.empty(n, dtype=torch.int64, pin_memory=True)
    ho_v = torch.empty(n, dtype=torch.float64, pin_memory=True)
    dk_a, dv_a, dk_b, dv_b = (torch.empty_like(t, device=dev) for t in (hk_a, hv_a, hk_b, hv_b))

    def e2e_step():
        dk_a.copy_(hk_a, non_blocking=True)
        dv_a.copy_(hv_a, non_blocking=True)
        dk_b.copy_(hk_b, non_blocking=True)
        dv_b.copy_(hv_b, non_blocking=True)
        L.sort_reduce(dk_a, dv_a, dk_b, dv_b, max_key=MAX_KEY, a_rekey=spec, out_keys=out_k, out_vals=out_v,
                      count=cnt, ws=ws, sync=False)
        m = int(cnt.item())  # the caller learns the result size, then copies the result
        ho_k[:m].copy_(out_k[:m], non_blocking=True)
        ho_v[:m].copy_(out_v[:m], non_blocking=True)
        return m

    e2e_steps = max(3, min(args.steps, 10))
    e2e_step()
    torch.cuda.synchronize()
    barrier(world)
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    for _ in range(e2e_steps):
        m = e2e_step()
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1) / e2e_steps, world)
    e2e_value = n * world / (e2e_ms * 1e-3)

    # ---- roofline of the dominant kernel (one onesweep digit pass) --------
    peak, peak_kind = peaks()
    avg_ms = os_ms / max(os_launches, 1)
    alg_bytes = 32.0 * n  # read 16 B + write 16 B per pair per pass
    achieved = alg_bytes / (avg_ms * 1e-3) / 1e9
    tpp = profile_traffic("sort_onesweep_merge_512x4_2x64M")
    roofline = {"bound": "hbm", "kernel": "sort_onesweep (one 9-bit LSD digit pass over 2^27 (u64,f64) pairs)",
                "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                "peak_source": f"{peak_kind} (MEASURED_PEAKS.json hbm_gbs)" if peak_kind == "measured" else peak_kind,
                "alg_bytes_per_launch": alg_bytes, "avg_launch_ms": avg_ms,
                "traffic": (tpp * n) if tpp else None}
    step_alg = 16.0 * n + 16.0 * n_out
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
            "config": {"workload": WORKLOAD, "nnz_per_operand": NNZ, "output_nnz": n_out,
                       "l2": "inputs (2 GiB) and sort buffers larger than the 126 MB L2; no flush needed",
                       "parallelism": f"replicas x{world}" if world > 1 else "1 GPU"},
            "e2e": {"value": e2e_value, "unit": "nnz/s", "ms_per_step": e2e_ms,
                    "h2d_bytes_per_step": int(16 * n), "d2h_bytes_per_step": int(16 * m + 8)},
            "gpu_launches": launches,
            "step_alg_bytes": step_alg, "step_hbm_frac_alg": step_alg / (ms * 1e-3) / 1e9 / peak,
            "kernels": kernels,
            "roofline": roofline,
            "cpu_baseline": cpu,
            "clocks": sampler.summary(),
        }
        print(json.dumps(result), flush=True)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


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
    args = ap.parse_args()
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

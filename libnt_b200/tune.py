"""Autotuner for the library's kernel choices.

* ``--sort`` (the default when no section is named): times every compiled
  onesweep variant (digit width, CTA size, items per thread, look-back window;
  listed by ``lnt_sort_variant_count``/``lnt_sort_variant``) over a grid of
  (pair count, key width) cases and keeps the fastest per case;
* ``--pass8``: the digit-pass shape of the bucketed sort + collect, timed on a
  2 x 2^24-pair merge under a four-mode permutation (LNT_PASS8_VARIANT);
* ``--batched``: the work-queue chunk (units per grab, the segment split) of the
  batched contraction engine, timed on 1024 problems drawn like the batched
  workload (dims U{16..512}, nnz log-uniform in [1e2, 1e5]) (LNT_BATCH_CHUNK);
* ``--tile``: the dense-row threshold divisor of the tile engine, timed on a
  reduced skewed contraction (LNT_TILE_DENSE_DIV).

Results are merged into ``csrc/lnt_tuned.json`` and the header
``csrc/lnt_tuned.h`` that the library compiles in is regenerated from it
(``--write``).  Rebuild afterwards (``python -m libnt_b200.build``).

    python -m libnt_b200.tune [--sort] [--pass8] [--batched] [--tile] [--write] [--quick]
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
TUNED_H = PKG / "csrc" / "lnt_tuned.h"
TUNED_JSON = PKG / "csrc" / "lnt_tuned.json"

KEY_BITS = [16, 24, 32, 36, 40, 48, 63]
LOG_N = [14, 17, 20, 23, 26, 27]


def variants(L):
    import ctypes as C
    lib = L.lib()
    out = []
    for i in range(lib.lnt_sort_variant_count()):
        b, t, it, w = C.c_int(), C.c_int(), C.c_int(), C.c_int()
        lib.lnt_sort_variant(i, C.byref(b), C.byref(t), C.byref(it), C.byref(w))
        out.append({"index": i, "bits": b.value, "threads": t.value, "items": it.value, "window": w.value})
    return out


def time_sort(L, torch, n, key_bits, variant, reps=5):
    os.environ["LNT_SORT_VARIANT"] = str(variant)
    g = torch.Generator(device="cuda")
    g.manual_seed(n + key_bits)
    hi = min(2 ** key_bits, 2 ** 63 - 1)
    k = torch.randint(0, hi, (n,), generator=g, device="cuda", dtype=torch.int64)
    v = torch.rand(n, generator=g, device="cuda", dtype=torch.float64)
    ok, ov = torch.empty_like(k), torch.empty_like(v)
    ws = L.workspace(L.sort_pairs_workspace(n, 2 ** key_bits))
    ts = []
    for r in range(reps + 2):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        L.sort_pairs(k, v, max_key=2 ** key_bits, out_keys=ok, out_vals=ov, ws=ws)
        e1.record()
        torch.cuda.synchronize()
        if r >= 2:
            ts.append(e0.elapsed_time(e1))
    if L.device_status() != 0:
        raise RuntimeError(f"device wait expired for variant {variant}")
    return statistics.median(ts)


def load_tuned() -> dict:
    if TUNED_JSON.exists():
        return json.loads(TUNED_JSON.read_text())
    return {"sort": [], "pass8_variant": 0, "batch_chunk": 8, "tile_dense_div": 8}


def render_header(tuned: dict) -> str:
    """Text of csrc/lnt_tuned.h for the tuned values."""
    lines = [
        "// Autotuned kernel choices.  Written by libnt_b200/tune.py from timings on a",
        "// B200 (the values come from lnt_tuned.json); sort entries are tried in",
        "// order, the first whose ranges contain the request wins.  An empty table",
        "// falls back to the untuned default.",
        "#pragma once",
        "",
        "namespace lnt {",
        "",
        "struct TunedSortEntry {",
        "  int key_bits_max;             // request key width <= this",
        "  unsigned long long n_max;     // request pair count <= this",
        "  int variant;                  // index into the compiled onesweep variants",
        "};",
        "",
        "static const TunedSortEntry kTunedSort[] = {",
    ]
    for e in tuned["sort"]:
        lines.append(f"    {{{e['key_bits_max']}, {e['n_max']}ull, {e['variant']}}},  "
                     f"// {e['ms']:.3f} ms at n=2^{e['log_n']}, {e['key_bits']} bits")
    lines += [
        "};",
        "",
        "// digit-pass shape of the bucketed sort + collect (see run_onesweep_pass8)",
        f"constexpr int kTunedPass8Variant = {int(tuned['pass8_variant'])};",
        "// bucket geometry of the sort merge (0: 2^(lg n - 12) buckets, 1: 2^(lg n - 11))",
        f"constexpr int kTunedBucketSmall = {int(tuned.get('bucket_small', 0))};",
        "// work-queue chunk of the batched contraction engine (units per grab)",
        f"constexpr unsigned kTunedBatchChunk = {int(tuned['batch_chunk'])};",
        "// dense-row threshold divisor of the tile engine",
        f"constexpr int kTunedTileDenseDiv = {int(tuned['tile_dense_div'])};",
        "",
        "}  // namespace lnt",
        "",
    ]
    return "\n".join(lines)


def write_header(tuned: dict):
    TUNED_H.write_text(render_header(tuned))


def _events(torch):
    return torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)


def _median_ms(torch, fn, reps=5, warm=2):
    ts = []
    for r in range(reps + warm):
        e0, e1 = _events(torch)
        e0.record()
        fn()
        e1.record()
        torch.cuda.synchronize()
        if r >= warm:
            ts.append(e0.elapsed_time(e1))
    return statistics.median(ts)


def tune_pass8(L, torch, quick=False):
    """Bucketed sort + collect of a 2 x 2^24-pair merge (keys < 512^4, A re-keyed
    by the reversal permutation), per LNT_PASS8_VARIANT."""
    n = 1 << (23 if quick else 24)
    g = torch.Generator(device="cuda")
    g.manual_seed(7)
    mk = 512 ** 4
    ak = torch.randint(0, mk, (n,), generator=g, device="cuda")
    bk = torch.randint(0, mk, (n,), generator=g, device="cuda")
    av = torch.rand(n, generator=g, device="cuda", dtype=torch.float64)
    bv = torch.rand(n, generator=g, device="cuda", dtype=torch.float64)
    spec = L.RekeySpec.make([512] * 4, [0, 1, 2, 3], [3, 2, 1, 0])
    ok = torch.empty(2 * n, dtype=torch.int64, device="cuda")
    ov = torch.empty(2 * n, dtype=torch.float64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ws = L.workspace(L.sort_reduce_workspace(n, n, mk))
    res = {}
    for v in range(4):
        os.environ["LNT_PASS8_VARIANT"] = str(v)
        res[v] = _median_ms(torch, lambda: L.sort_reduce(ak, av, bk, bv, max_key=mk, a_rekey=spec, out_keys=ok,
                                                          out_vals=ov, count=cnt, ws=ws, sync=False))
        print(f"pass8 variant {v}: {res[v]:.3f} ms", flush=True)
    os.environ.pop("LNT_PASS8_VARIANT", None)
    return min(res, key=res.get), res


def tune_bucket(L, torch, quick=False):
    """The merge of tune_pass8 at 2 x 2^26 pairs (2^25 with --quick) with the
    large and the small bucket geometry (LNT_BUCKET_SMALL)."""
    n = 1 << (25 if quick else 26)
    g = torch.Generator(device="cuda")
    g.manual_seed(11)
    mk = 512 ** 4
    ak = torch.randint(0, mk, (n,), generator=g, device="cuda")
    bk = torch.randint(0, mk, (n,), generator=g, device="cuda")
    av = torch.rand(n, generator=g, device="cuda", dtype=torch.float64)
    bv = torch.rand(n, generator=g, device="cuda", dtype=torch.float64)
    spec = L.RekeySpec.make([512] * 4, [0, 1, 2, 3], [3, 2, 1, 0])
    ok = torch.empty(2 * n, dtype=torch.int64, device="cuda")
    ov = torch.empty(2 * n, dtype=torch.float64, device="cuda")
    cnt = torch.zeros(1, dtype=torch.int64, device="cuda")
    ws = L.workspace(L.sort_reduce_workspace(n, n, mk))
    res = {}
    for small in (0, 1):
        os.environ["LNT_BUCKET_SMALL"] = str(small)
        res[small] = _median_ms(torch, lambda: L.sort_reduce(ak, av, bk, bv, max_key=mk, a_rekey=spec, out_keys=ok,
                                                              out_vals=ov, count=cnt, ws=ws, sync=False))
        print(f"bucket geometry small={small}: {res[small]:.3f} ms", flush=True)
    os.environ.pop("LNT_BUCKET_SMALL", None)
    return min(res, key=res.get), res


def batch_problems(count, seed=0):
    """count problems a(i,j,k)*b(k,l,j) as lattices: dims U{16..512}, nnz
    log-uniform in [1e2, 1e5] clamped to the lattice size, key-sorted sets."""
    import numpy as np
    dims, ak, bk = [], [], []
    for p in range(count):
        r = np.random.default_rng([seed, p])
        i, j, k, l = (int(x) for x in r.integers(16, 513, 4))
        h, w, wB = i, j * k, l
        na = min(int(round(10 ** r.uniform(2, 5))), h * w)
        nb = min(int(round(10 ** r.uniform(2, 5))), w * wB)
        ak.append(np.unique(r.integers(0, h * w, int(na * 1.1) + 8, dtype=np.uint64))[:na])
        bk.append(np.unique(r.integers(0, w * wB, int(nb * 1.1) + 8, dtype=np.uint64))[:nb])
        dims.append((h, w, wB, 1))
    return dims, ak, bk


def tune_batched(L, torch, quick=False):
    import numpy as np
    dims, ak, bk = batch_problems(256 if quick else 1024)
    a_off = np.concatenate([[0], np.cumsum([x.size for x in ak])]).astype(np.uint64)
    b_off = np.concatenate([[0], np.cumsum([x.size for x in bk])]).astype(np.uint64)
    akd = torch.from_numpy(np.concatenate(ak).view(np.int64)).cuda()
    bkd = torch.from_numpy(np.concatenate(bk).view(np.int64)).cuda()
    avd = torch.rand(akd.numel(), device="cuda", dtype=torch.float64) * 2 - 1
    bvd = torch.rand(bkd.numel(), device="cuda", dtype=torch.float64) * 2 - 1
    res = {}
    for c in (1, 2, 4, 8, 16, 32, 64):
        os.environ["LNT_BATCH_CHUNK"] = str(c)
        batch = L.Batch(np.array(dims, np.int64), a_off, b_off, akd, avd, bkd, bvd)
        res[c] = _median_ms(torch, batch.run)
        print(f"batch chunk {c}: {res[c]:.3f} ms", flush=True)
        del batch
    os.environ.pop("LNT_BATCH_CHUNK", None)
    return min(res, key=res.get), res


def tune_tile(L, torch, quick=False):
    """Skewed contraction c(i,j,m) = a(i,j,k,l) * b(k,l,m), a 128x128x256x256 with
    2^19 coordinates (32 per output row), b 256x256x4096 with 2^25 (24 with
    --quick), (k,l) Zipf(1.1) aligned: the tile engine, per LNT_TILE_DENSE_DIV."""
    g = torch.Generator(device="cuda")
    g.manual_seed(0)
    di, dj, dk, dl, dm = 128, 128, 256, 256, 4096

    def zipf(n, dim):
        p = torch.arange(1, dim + 1, dtype=torch.float64, device="cuda") ** -1.1
        cdf = torch.cumsum(p / p.sum(), 0)
        return torch.searchsorted(cdf, torch.rand(n, generator=g, device="cuda", dtype=torch.float64)).clamp_(
            max=dim - 1)

    na, nb = 1 << 19, 1 << (24 if quick else 25)
    ak = torch.unique(torch.randint(0, di, (na,), generator=g, device="cuda")
                      + di * torch.randint(0, dj, (na,), generator=g, device="cuda")
                      + (di * dj) * (zipf(na, dk) + dk * zipf(na, dl)))
    bk = torch.unique(zipf(nb, dk) + dk * zipf(nb, dl) + (dk * dl) * torch.randint(0, dm, (nb,), generator=g,
                                                                                    device="cuda"))
    av = torch.randn(ak.numel(), generator=g, device="cuda", dtype=torch.float64)
    bv = torch.randn(bk.numel(), generator=g, device="cuda", dtype=torch.float64)
    res = {}
    for dv in (2, 4, 8, 16, 32):
        os.environ["LNT_TILE_DENSE_DIV"] = str(dv)
        os.environ["LNT_SPGEMM_ENGINE"] = "tile"
        res[dv] = _median_ms(torch, lambda: L.lattice_mult(ak, av, bk, bv, di * dj, dk * dl, dm, 1), reps=3, warm=1)
        print(f"tile dense divisor {dv}: {res[dv]:.3f} ms", flush=True)
    os.environ.pop("LNT_TILE_DENSE_DIV", None)
    os.environ.pop("LNT_SPGEMM_ENGINE", None)
    return min(res, key=res.get), res


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--sort", action="store_true", help="onesweep variant table")
    ap.add_argument("--pass8", action="store_true", help="digit-pass shape of the bucketed sort + collect")
    ap.add_argument("--bucket", action="store_true", help="bucket geometry of the sort merge")
    ap.add_argument("--batched", action="store_true", help="work-queue chunk of the batched engine")
    ap.add_argument("--tile", action="store_true", help="dense-row divisor of the tile engine")
    ap.add_argument("--write", action="store_true", help="merge into csrc/lnt_tuned.json and rewrite csrc/lnt_tuned.h")
    ap.add_argument("--quick", action="store_true", help="fewer and smaller cases")
    ap.add_argument("--json", default=None, help="also dump the raw timings here")
    args = ap.parse_args()
    if not (args.sort or args.pass8 or args.bucket or args.batched or args.tile):
        args.sort = True
    sys.path.insert(0, str(PKG.parent))
    import torch

    import libnt_b200 as L
    tuned = load_tuned()
    raw = {}
    if args.sort:
        vs = variants(L)
        kb_list = [24, 36, 63] if args.quick else KEY_BITS
        ln_list = [20, 27] if args.quick else LOG_N
        results, best = [], []
        for kb in kb_list:
            for ln in ln_list:
                n = 1 << ln
                row = {"key_bits": kb, "log_n": ln, "ms": {}}
                for v in vs:
                    row["ms"][v["index"]] = time_sort(L, torch, n, kb, v["index"])
                win = min(row["ms"], key=row["ms"].get)
                results.append(row)
                passes = -(-kb // vs[win]["bits"])
                print(f"bits={kb:2d} n=2^{ln:2d} best variant {win} {vs[win]} {row['ms'][win]:.3f} ms "
                      f"({passes} passes, {32 * n * passes / row['ms'][win] / 1e6:.0f} GB/s per-pass-bytes)",
                      flush=True)
                best.append({"key_bits_max": kb, "n_max": n if ln != ln_list[-1] else 2 ** 62, "variant": win,
                             "ms": row["ms"][win], "log_n": ln, "key_bits": kb})
        os.environ.pop("LNT_SORT_VARIANT", None)
        tuned["sort"] = best
        raw["sort"] = {"variants": vs, "results": results}
    if args.pass8:
        tuned["pass8_variant"], raw["pass8"] = tune_pass8(L, torch, args.quick)
    if args.bucket:
        tuned["bucket_small"], raw["bucket"] = tune_bucket(L, torch, args.quick)
    if args.batched:
        tuned["batch_chunk"], raw["batched"] = tune_batched(L, torch, args.quick)
    if args.tile:
        tuned["tile_dense_div"], raw["tile"] = tune_tile(L, torch, args.quick)
    print("tuned:", {k: v for k, v in tuned.items() if k != "sort"})
    if args.json:
        Path(args.json).write_text(json.dumps(raw, indent=1, default=str))
    if args.write:
        TUNED_JSON.write_text(json.dumps(tuned, indent=1) + "\n")
        write_header(tuned)
        print("wrote", TUNED_JSON, "and", TUNED_H)


if __name__ == "__main__":
    main()

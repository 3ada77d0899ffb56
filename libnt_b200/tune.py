"""Autotuner for the onesweep radix sort.

Times every compiled kernel variant (digit width, CTA size, items per thread,
look-back window; listed by ``lnt_sort_variant_count``/``lnt_sort_variant``)
on the current GPU over a grid of (pair count, key width) cases, picks the
fastest per case and writes the table ``csrc/lnt_tuned.h`` that the library
compiles in.  Rebuild afterwards (``python -m libnt_b200.build``).

    python -m libnt_b200.tune [--write] [--quick] [--json results.json]
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


def write_header(best: list[dict]):
    lines = [
        "// Autotuned kernel choices.  Written by libnt_b200/tune.py from timings on a",
        "// B200; entries are tried in order, the first whose ranges contain the",
        "// request wins.  An empty table falls back to the untuned default.",
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
    for e in best:
        lines.append(f"    {{{e['key_bits_max']}, {e['n_max']}ull, {e['variant']}}},  "
                     f"// {e['ms']:.3f} ms at n=2^{e['log_n']}, {e['key_bits']} bits")
    lines += ["};", "", "}  // namespace lnt", ""]
    TUNED_H.write_text("\n".join(lines))


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--write", action="store_true", help="write csrc/lnt_tuned.h")
    ap.add_argument("--quick", action="store_true", help="fewer cases")
    ap.add_argument("--json", default=None)
    args = ap.parse_args()
    sys.path.insert(0, str(PKG.parent))
    import torch

    import libnt_b200 as L
    vs = variants(L)
    kb_list = [24, 36, 63] if args.quick else KEY_BITS
    ln_list = [20, 27] if args.quick else LOG_N
    results = []
    best = []
    prev_kb = 0
    for kb in kb_list:
        prev_n = 0
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
            prev_n = n
        prev_kb = kb
    os.environ.pop("LNT_SORT_VARIANT", None)
    if args.json:
        Path(args.json).write_text(json.dumps({"variants": vs, "results": results}, indent=1))
    if args.write:
        write_header(best)
        print("wrote", TUNED_H)


if __name__ == "__main__":
    main()

"""Autotune this library's launch shapes on the current GPU and write the
table that Context.load_tuning applies (bench.py loads
p3-miden_b200/tuning/<device>.json when it exists).

    python p3-miden_b200/autotune.py [--out p3-miden_b200/tuning/b200.json]

Tuned: the bit-range split of the coset LDE for the transform heights of the
measured workloads (the headline Keccak slabs, the quotient chunks, the
lifted cubic traces and FRI-sized transforms), and the column-slab width of
the main commit of the headline trace. Every choice computes the same values;
only the time changes.
"""
from __future__ import annotations

import argparse
import importlib.util
import json
import sys
from pathlib import Path

HERE = Path(__file__).resolve().parent

# (log_h, width, log_blowup): main-trace slabs of the 2^18 x 2633 Keccak trace
# (336 columns), its quotient chunks (4 columns), the lifted cubic traces
# (blowup 8) and the batch mix's heights.
LDE_SHAPES = [(18, 336, 1), (18, 4, 1), (20, 64, 3), (16, 256, 3), (12, 1024, 3), (14, 128, 3), (17, 64, 3),
              (15, 336, 3), (13, 336, 3)]
SLAB_SHAPES = [(18, 2633, 1)]


def load_product():
    spec = importlib.util.spec_from_file_location("p3_miden_b200", HERE / "__init__.py",
                                                  submodule_search_locations=[str(HERE)])
    mod = importlib.util.module_from_spec(spec)
    sys.modules["p3_miden_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--out", default=str(HERE / "tuning" / "b200.json"))
    ap.add_argument("--reps", type=int, default=3)
    args = ap.parse_args()
    import torch
    P = load_product()
    ctx = P.Context(0)
    table = {"device": torch.cuda.get_device_name(0), "lde_split": {}, "slab_cols": 0, "measurements": []}
    seen = set()
    for log_h, w, lb in LDE_SHAPES:
        r = ctx.autotune_lde(log_h, w, lb, args.reps)
        table["measurements"].append(r)
        print(json.dumps(r), flush=True)
        if log_h not in seen:  # the first (most important) shape of each height decides
            table["lde_split"][str(log_h)] = r["split"]
            seen.add(log_h)
            ctx.set_lde_split(log_h, r["split"])
    for log_h, w, lb in SLAB_SHAPES:
        r = ctx.autotune_slabs(log_h, w, lb, 2)
        table["measurements"].append(r)
        print(json.dumps(r), flush=True)
        table["slab_cols"] = r["slab_cols"]
    ctx.close()
    Path(args.out).parent.mkdir(parents=True, exist_ok=True)
    Path(args.out).write_text(json.dumps(table, indent=1) + "\n")
    print(f"wrote {args.out}")


if __name__ == "__main__":
    main()

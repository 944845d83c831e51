"""Generate tests/golden/golden.json -- run in a container that has the reference.

Each case is a seeded synthetic matrix with the shape and value distribution of
one workload (no reference data file is copied).  Expected values:
  exact      -- multi-modular exact integer permanent (integer matrices)
  dd         -- double-double Gray-code Ryser (hi, lo)
  dp         -- subset dynamic programme in __float128 (n <= 22)
  ref_*      -- the reference's own functions, compiled from its sources
                (oracle/_ref/libperman_ref.so), at full double precision
Usage: python tests/golden/make_golden.py [--big] [--huge] [--only NAME ...]
  --huge adds the full-size SkipPer configuration (n=36, density 0.20, values
  U(0,1]; about 20 minutes on 8 cores); --only recomputes the named cases and
  merges them into the existing file.
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT / "oracle"))
from oracle import Oracle, Reference  # noqa: E402

THREADS = os.cpu_count() or 8


def bernoulli(rng, n, d):
    while True:
        m = (rng.random((n, n)) < d).astype(np.float64)
        if m.any(axis=0).all() and m.any(axis=1).all():
            return m


def cfg2_n36_matrix():
    """The sparse exact configuration at full size: n=36, Bernoulli(0.20) mask
    (no empty row or column), nonzero values 1 - U[0,1) = U(0,1], seed 2026 --
    the same instance bench.py's secondary workload uses."""
    rng = np.random.default_rng(2026)
    while True:
        mk = rng.random((36, 36)) < 0.2
        if mk.any(0).all() and mk.any(1).all():
            break
    return mk * (1.0 - rng.random((36, 36)))


def make_cases(big: bool, huge: bool = False):
    cases = []
    rng = np.random.default_rng(20261203)
    # small mixed cases (every n from 1 to 20, all three types)
    for n in range(1, 21):
        kind = ["binary", "int", "real"][n % 3]
        m = bernoulli(rng, n, 0.6) if n > 1 else np.ones((1, 1))
        if kind == "int":
            m = m * rng.integers(1, 6, (n, n))
        elif kind == "real":
            m = m * (1.0 - rng.random((n, n)))
        cases.append((f"small_{kind}_{n}", kind, m))
    # signed integer and signed real matrices (cancellation)
    cases.append(("signed_int_16", "int", rng.integers(-3, 4, (16, 16)).astype(np.float64)))
    cases.append(("signed_real_14", "real", rng.standard_normal((14, 14))))
    # configuration-shaped cases
    cases.append(("cfg1_binary_n30_d050", "binary", bernoulli(np.random.default_rng(101), 30, 0.5)))
    r2 = np.random.default_rng(202)
    m2 = bernoulli(r2, 28, 0.20) * (1.0 - r2.random((28, 28)))
    cases.append(("cfg2_sparse_real_n28_d020", "real", m2))
    r3 = np.random.default_rng(303)
    m3 = bernoulli(r3, 24, 0.5) * r3.integers(1, 5, (24, 24))
    cases.append(("cfg3_int_n24_d050", "int", m3))
    if big:
        r4 = np.random.default_rng(304)
        m4 = bernoulli(r4, 32, 0.5) * r4.integers(1, 5, (32, 32))
        cases.append(("cfg3_int_n32_d050", "int", m4))
        r5 = np.random.default_rng(505)
        m5 = bernoulli(r5, 30, 0.5) * (1.0 - r5.random((30, 30)))
        cases.append(("real_n30_d050", "real", m5))
    if huge:
        cases.append(("cfg2_sparse_real_n36_d020", "real", cfg2_n36_matrix()))
    return cases


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--big", action="store_true", help="include the n=30/32 cases (minutes)")
    ap.add_argument("--huge", action="store_true", help="include the n=36 SkipPer case (about 20 minutes)")
    ap.add_argument("--only", nargs="*", default=None, help="recompute these cases, keep the others")
    ap.add_argument("--out", default=str(Path(__file__).with_name("golden.json")))
    args = ap.parse_args()
    orc = Oracle()
    ref = Reference()
    out = []
    kept = {}
    if args.only and Path(args.out).exists():
        kept = {c["name"]: c for c in json.load(open(args.out))["cases"]}
    for name, kind, m in make_cases(args.big, args.huge):
        if args.only is not None and name not in args.only:
            if name in kept:
                out.append(kept[name])
            continue
        n = m.shape[0]
        t0 = time.time()
        rec = {"name": name, "kind": kind, "n": n, "matrix": m.tolist()}
        hi, lo = orc.perm_dd(m, THREADS)
        rec["dd"] = [hi, lo]
        if n <= 22:
            rec["dp"] = list(orc.perm_dp(m))
        if kind in ("binary", "int"):
            exact, _ = orc.perm_exact_int(m.astype(np.int64), THREADS)
            rec["exact"] = str(exact)
        rec["ref_perman64"] = ref.perman64(m) if n <= 30 else None
        rec["ref_parallel_perman64"] = ref.parallel_perman64(m, THREADS)
        rec["threads"] = THREADS
        if n >= 2:
            c = ref.compress(2, m)
            t1 = time.time()
            rec["ref_skip_balanced_skiporder"] = ref.skip_balanced(c, THREADS)
            rec["ref_skip_seconds"] = round(time.time() - t1, 2)
        rec["seconds"] = round(time.time() - t0, 2)
        print(name, n, rec.get("exact", rec["dd"][0]), f"{rec['seconds']}s", flush=True)
        out.append(rec)
    names = {c["name"] for c in out}
    out.extend(c for name, c in kept.items() if name not in names)
    with open(args.out, "w") as f:
        json.dump({"generator": "tests/golden/make_golden.py", "cases": out}, f, indent=None)
        f.write("\n")
    print("wrote", args.out)


if __name__ == "__main__":
    main()

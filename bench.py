"""Benchmark: dense exact Ryser permanent, n=40, density 0.5, values U{1,2,3,4}.

One step = one whole exact permanent (2^39 Gray steps x 2n FP64 operations)
of a seeded synthetic matrix that is already resident in device memory;
`value` is Ryser Gray steps per second.  With N ranks (torchrun, one GPU
each) the one matrix is sharded: rank r walks Gray-range shard r of N
(perm_exact_dense_resident_shard) and the 16-byte (hi, lo) partials are
all-gathered over NCCL and added in double-double (strong scaling; at N=1
the step is the whole walk).  A weak-scaling secondary (every rank its own
matrix) is kept beside it.  `e2e` is the same metric through the C-ABI
call with a host matrix (host->device copy and result readback inside the
timed region).  `roofline` relates the kernel's algorithmic FP64 operations to
the FP64 peak measured live on the same chip; `cpu_baseline` is the
reference's own CPU Ryser (compiled from its sources into oracle/_ref) on a
bounded Gray-range sample of the same matrix, with every host core.

python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
"""
from __future__ import annotations

import argparse
import ctypes
import hashlib
import importlib.util
import json
import os
import statistics
import subprocess
import sys
import time
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parent
PKG = ROOT / "matrix-permanent-calculator_b200"
N_ORDER = 40
DENSITY = 0.5
SEED = 303
METRIC = "Ryser Gray steps/s (dense exact permanent, FP64)"
WORKLOAD = "dense exact Ryser, n=40, density 0.5, values U{1,2,3,4}"


def load_pkg():
    spec = importlib.util.spec_from_file_location("perman_b200", PKG / "__init__.py")
    mod = importlib.util.module_from_spec(spec)
    sys.modules["perman_b200"] = mod
    spec.loader.exec_module(mod)
    return mod


def make_matrix(rank: int, n: int = N_ORDER, d: float = DENSITY) -> np.ndarray:
    rng = np.random.default_rng(SEED + 1000 * rank)
    while True:
        m = rng.random((n, n)) < d
        if m.any(axis=0).all() and m.any(axis=1).all():
            break
    return (m * rng.integers(1, 5, (n, n))).astype(np.int32)


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


class Clocks:
    """nvidia-smi sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        self.lines = []
        if self.proc:
            self.proc.terminate()
            try:
                out, _ = self.proc.communicate(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
                out, _ = self.proc.communicate()
            self.lines = [l for l in out.splitlines() if l.strip()]

    def summary(self):
        sm, mx, reasons = [], 0.0, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for l in getattr(self, "lines", []):
            f = [x.strip() for x in l.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = max(mx, float(f[2]))
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"], "samples": 0}
        load = [s for s in sm if s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx, "reasons": sorted(reasons), "samples": len(sm)}


def flush_l2(buf):
    if buf is not None:
        buf.add_(1.0)


def cpu_reference_rate(A: np.ndarray, target_s: float, threads: int):
    """Reference cpu_perman64 (gpu_exact_dense.cu:7) over a Gray sub-range of the
    same n=40 workload: returns (steps/s, steps, seconds)."""
    sys.path.insert(0, str(ROOT / "oracle"))
    from oracle import Reference

    ref = Reference()
    Ad = A.astype(np.float64)
    probe = 1 << 24
    t = time.perf_counter()
    ref.cpu_perman64_range(Ad, 1, 1 + probe, threads)
    dt = time.perf_counter() - t
    steps = int(min(1 << 36, max(probe, probe * target_s / max(dt, 1e-6))))
    t = time.perf_counter()
    ref.cpu_perman64_range(Ad, 1, 1 + steps, threads)
    dt = time.perf_counter() - t
    return steps / dt, steps, dt


def run_reference_arm(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    threads = os.cpu_count() or 1
    A = make_matrix(0)
    try:
        sys.path.insert(0, str(ROOT / "oracle"))
        from oracle import Reference

        ref = Reference()
    except Exception as e:  # pragma: no cover - reported, not raised
        print(json.dumps({"impl": "reference", "unavailable": f"reference CPU build missing: {e}"}))
        return 0
    Ad = A.astype(np.float64)
    # size one step (a Gray sub-range) so that the whole run stays within minutes
    rate0, _, _ = cpu_reference_rate(A, 1.0, threads)
    steps_per = int(max(1 << 22, min(1 << 34, rate0 * 3.0)))
    for _ in range(args.warmup):
        ref.cpu_perman64_range(Ad, 1, 1 + steps_per, threads)
    times = []
    for k in range(args.steps):
        start = 1 + k * steps_per
        t = time.perf_counter()
        ref.cpu_perman64_range(Ad, start, start + steps_per, threads)
        times.append(time.perf_counter() - t)
    total = sum(times)
    value = steps_per * args.steps / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / args.steps,
        "higher_is_better": True, "scaling": "strong", "vs_baseline": None, "dtype": "f64",
        "data": "synthetic (seeded)",
        "config": {"workload": WORKLOAD, "sample": f"Gray indices [1+k*{steps_per}, 1+(k+1)*{steps_per}) per step",
                   "function": "cpu_perman64 (gpu_exact_dense.cu:7), OpenMP"},
        "cpu_baseline": {"value": value, "unit": "steps/s", "cores": threads, "kind": "reference",
                         "sample": f"{steps_per} Gray steps of the n=40 walk per step"},
        "e2e": {"value": value, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


# Sources whose text determines each profiled kernel's instruction stream:
# a recorded ncu count is only valid for the same template instance compiled
# from the same text.
KERNEL_SOURCES = {
    "int32x": ["ryser_dense_int_sparse.cuh", "ryser_dense_int.cuh", "ryser_dense.cuh", "perman_common.cuh"],
    "fp64x": ["ryser_dense_2l.cuh", "ryser_dense.cuh", "perman_common.cuh"],
    "int32x_dd": ["ryser_dense_intc_sparse.cuh", "ryser_dense_intc.cuh", "ryser_dense_int_sparse.cuh",
                  "ryser_dense_int.cuh", "ryser_dense.cuh", "perman_common.cuh"],
}


def source_sha16(kname: str) -> str | None:
    files = KERNEL_SOURCES.get(kname)
    if not files:
        return None
    h = hashlib.sha256()
    for f in files:
        h.update((PKG / "csrc" / f).read_bytes())
    return h.hexdigest()[:16]


def kernel_template(kname: str, A: np.ndarray) -> str:
    n = A.shape[0]
    if kname == "int32x":
        g, ngo, ng1, ng2 = (sys.modules.get("perman_b200") or load_pkg()).int_layout(A)
        if ng1:
            return f"ryser_dense_int_3l_kernel<{n}, {g}, {ng1}, {ng2}>"
        return f"ryser_dense_int_sparse_kernel<{n}, {g}, {ngo}>" if ngo else f"ryser_dense_int_kernel<{n}, {g}>"
    if kname == "int32x_dd":
        # product groups and pairing as the engine lays them out; last template
        # argument: CTAs per SM compiled for (3 up to order 36, 2 above)
        g, pair, ngo, ng1, ng2 = (sys.modules.get("perman_b200") or load_pkg()).intc_layout(A)
        pb_ = "true" if pair else "false"
        if ng1:
            return f"ryser_dense_intc_3l_kernel<{n}, {g}, {pb_}, {ng1}, {ng2}, {3 if n <= 40 else 2}>"
        if ngo:
            return f"ryser_dense_intc_sparse_kernel<{n}, {g}, {pb_}, {ngo}, {3 if n <= 36 else 2}>"
        return f"ryser_dense_intc_kernel<{n}, {g}, {pb_}, {3 if n <= 36 else 2}>"
    if kname == "fp64x":
        r1, r = (sys.modules.get("perman_b200") or load_pkg()).fp64_levels(A)
        if r1:
            return f"ryser_dense_3l_kernel<{n}, {r1}, {r}>"
        return f"ryser_dense_2l_kernel<{n}, {r}>" if r else f"ryser_dense_kernel<{n}>"
    return kname


def load_profile(kname: str, A: np.ndarray) -> tuple[dict | None, str | None]:
    """ncu figures of one launch of this kernel's template instance (profiles/),
    and why they do not apply (None when they do): recorded for another
    instance, or for other source text than this checkout's."""
    prof = ROOT / "profiles" / "ryser_dense_n40_issue.json"
    try:
        rec = json.loads(prof.read_text()).get(kname)
    except Exception:
        return None, "no profile record"
    if not rec:
        return None, "no profile record"
    want = kernel_template(kname, A)
    if rec.get("kernel") != want:
        return None, f"profile recorded for {rec.get('kernel')}, this run launches {want}"
    sha = source_sha16(kname)
    if rec.get("source_sha16") != sha:
        return rec, f"kernel sources changed since the profile (recorded {rec.get('source_sha16')}, now {sha})"
    return rec, None


def sharded_step(pb, shard_fn, rank: int, world: int, dist=None, device=None):
    """One step of the sharded workload: this rank's Gray-range shard of the
    one matrix (shard_fn(rank, world) -> (hi, lo, device ms)), then the
    16-byte all-gather of every rank's (hi, lo), added in rank order in
    double-double.  Returns ((hi, lo), device ms of the step on this rank:
    the shard's kernel plus the all-gather)."""
    hi, lo, ms = shard_fn(rank, world)
    parts = [(hi, lo)]
    if dist is not None and world > 1:
        import torch

        dev = f"cuda:{device}" if device is not None else "cpu"
        t = torch.tensor([hi, lo], dtype=torch.float64, device=dev)
        gathered = [torch.zeros_like(t) for _ in range(world)]
        if device is not None:
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            dist.all_gather(gathered, t)
            e1.record()
            e1.synchronize()
            ms += e0.elapsed_time(e1)
        else:
            t0 = time.perf_counter()
            dist.all_gather(gathered, t)
            ms += (time.perf_counter() - t0) * 1e3
        parts = [(float(g[0]), float(g[1])) for g in gathered]
    return pb.dd_sum(parts), ms


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-secondary", action="store_true")
    ap.add_argument("--order", type=int, default=N_ORDER, help="matrix order (profiling runs use a smaller one)")
    ap.add_argument("--workload", choices=["dense", "sparse"], default="dense",
                    help="dense: the n=40 U{1..4} headline matrix; sparse: the sparse exact configuration's "
                         "distribution (Bernoulli(0.2) mask, U(0,1] values, seed 2026) at --order, walked by "
                         "the certified split-dd kernel (profiling runs)")
    ap.add_argument("--variant", choices=["auto", "fp64", "int", "tc", "split", "intdd", "sdd"], default="auto",
                    help="dense kernel: automatic, FP64-X, int32-X, tensor-core row sums, split X or the "
                         "certified int32-X walk (double-double products and sum)")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference_arm(args)

    rank, world, local = dist_env()
    import torch

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    device = local if world > 1 else 0
    torch.cuda.set_device(device)
    pb = load_pkg()
    eng = pb.Engine(device)
    A = make_matrix(0, args.order) if args.workload == "dense" else cfg2_matrix(args.order)  # every rank shards it
    n = A.shape[0]
    variant = {"auto": 0, "fp64": pb.PERM_KERNEL_DENSE, "int": pb.PERM_KERNEL_DENSE_INT,
               "tc": pb.PERM_KERNEL_DENSE_TC, "split": pb.PERM_KERNEL_DENSE_SPLIT,
               "intdd": pb.PERM_KERNEL_DENSE_INT_DD, "sdd": pb.PERM_KERNEL_DENSE_SDD}[args.variant]
    if args.workload == "sparse" and variant == 0:
        variant = pb.PERM_KERNEL_DENSE_SDD  # the sparse configuration's automatic kernel
    total_steps = 2.0 ** (n - 1)
    ops_per_step = 2.0 * n  # n X-updates + n multiplies per Gray step (algorithmic)
    ops_text = f"2n = {int(ops_per_step)} FP64 ops per Gray step x 2^{n - 1} steps"
    if variant == pb.PERM_KERNEL_DENSE_SPLIT:
        # coarse and remainder X updates, a combine per entry, n - 1 multiplies
        ops_per_step = 4.0 * n - 1.0
        ops_text = f"4n - 1 = {int(ops_per_step)} FP64 ops per split-X Gray step x 2^{n - 1} steps"
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.float32, device=f"cuda:{device}")  # 256 MB > L2

    peak_ops, _ = eng.fp64_peak()
    peak_ops = max(peak_ops, eng.fp64_peak()[0])
    res = eng.upload_dense(A, variant=variant)
    if world > 1 and variant == pb.PERM_KERNEL_DENSE_TC:
        raise SystemExit("the tensor-core kernel runs whole walks only; use --variant int for sharded runs")

    def barrier():
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize(device)

    def resident_shard(r_, w_):
        rr = res.run_shard(r_, w_)
        resident_shard.last = rr
        return rr.hi, rr.lo, rr.kernel_ms

    for _ in range(args.warmup):
        sharded_step(pb, resident_shard, rank, world, dist, device)
        flush_l2(flush)
    barrier()
    kernel_ms, step_ms = [], []
    t0 = time.perf_counter()
    with Clocks(device) as clk:
        for _ in range(args.steps):
            flush_l2(flush)
            torch.cuda.synchronize(device)
            (hi, lo), ms = sharded_step(pb, resident_shard, rank, world, dist, device)
            kernel_ms.append(resident_shard.last.kernel_ms)
            step_ms.append(ms)
    barrier()
    wall = time.perf_counter() - t0
    r = resident_shard.last
    dev_s = sum(step_ms) * 1e-3
    if dist is not None:
        t = torch.tensor([dev_s], device=f"cuda:{device}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        dev_s = float(t.item())
    value = args.steps * total_steps / dev_s
    perm_value = r.value if world == 1 else hi + lo

    # end to end through the public C ABI with a host matrix: at N=1 the
    # reference-signature entry point gpu_perman64_xshared_coalescing_mshared_int
    # (upload, walk, double-double result back; one evaluation, like the
    # reference); at N>1 distributed_exact_dense (each rank uploads the host
    # matrix, walks its shard, the 16-byte partials are all-gathered)
    os.environ["PERM_DEVICE"] = str(device)
    plain = pb.Engine(device)
    plain.set_rel_target(-1.0)
    if world > 1:
        e2e_call = lambda: sum(pb.distributed_exact_dense(A, engine=plain))  # noqa: E731
        e2e_path = "distributed_exact_dense(): perm_exact_dense_shard() C ABI per rank with a host matrix + all-gather"
    elif variant == 0:
        shim = eng.lib.gpu_perman64_xshared_coalescing_mshared_int
        shim.restype = ctypes.c_double
        shim.argtypes = [ctypes.POINTER(ctypes.c_int), ctypes.c_int, ctypes.c_int, ctypes.c_int]
        A32 = np.ascontiguousarray(A, dtype=np.int32)
        e2e_call = lambda: shim(A32.ctypes.data_as(ctypes.POINTER(ctypes.c_int)), n, 2048, 256)  # noqa: E731
        e2e_path = "gpu_perman64_xshared_coalescing_mshared_int() C ABI (reference signature), host int32 matrix"
    else:
        e2e_call = lambda: plain.exact_dense(A, variant=variant).value  # noqa: E731
        e2e_path = "perm_exact_dense_ex() C ABI with a forced kernel, host matrix"
    e2e_ms = []
    for _ in range(2):
        e2e_call()
    barrier()
    for _ in range(args.steps):
        t = time.perf_counter()
        v2 = e2e_call()
        e2e_ms.append((time.perf_counter() - t) * 1e3)
    e2e_s = sum(e2e_ms) * 1e-3
    if dist is not None:
        t = torch.tensor([e2e_s], device=f"cuda:{device}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        e2e_s = float(t.item())
    assert v2 == perm_value, (v2, perm_value)  # same shards, deterministic reductions

    # weak scaling beside it: every rank its own matrix, one whole walk
    weak = None
    if world > 1:
        W = eng.upload_dense(make_matrix(rank, args.order), variant=variant)
        W.run()
        barrier()
        wms = W.run().kernel_ms
        W.free()
        t = torch.tensor([wms * 1e-3], device=f"cuda:{device}", dtype=torch.float64)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        weak = {"value": world * total_steps / float(t.item()), "unit": "steps/s",
                "ms_max_over_ranks": float(t.item()) * 1e3,
                "config": f"{world} ranks, one whole n={n} walk each (rank r: seed {SEED} + 1000 r)"}
        barrier()

    # the same matrix through perm_exact_dense with the accuracy policy
    # (target 1e-10): the certified walk for integer matrices
    policy = None
    if not args.no_secondary and rank == 0:
        eng.exact_dense(A, variant=variant)  # warm-up: first launch of the policy's kernel
        t = time.perf_counter()
        rp = eng.exact_dense(A, variant=variant)
        pms = (time.perf_counter() - t) * 1e3
        policy = {"ms": pms, "kernel_ms": rp.kernel_ms, "kernel": rp.kernel,
                  "rel_error_estimate": rp.rel_error_estimate,
                  "rel_diff_vs_single_evaluation": abs(rp.value - perm_value) / abs(perm_value),
                  "ratio_vs_single_evaluation_e2e": pms / (e2e_s * 1e3 / args.steps), "value": rp.value}
    barrier()

    mean_ms = statistics.mean(kernel_ms)
    achieved = (total_steps / world) * ops_per_step / (mean_ms * 1e-3)
    kname = {1: "fp64x", 3: "int32x", 5: "tc", 6: "splitx", 7: "int32x_dd"}.get(r.kernel, "")
    prof_rec, prof_stale = load_profile(kname, A)
    traffic = prof_rec.get("dram_bytes_per_launch") if prof_rec and not prof_stale else None

    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": dev_s * 1e3 / args.steps, "higher_is_better": True,
        "scaling": "strong", "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, resident in HBM)",
        "config": {"workload": (WORKLOAD.replace("n=40", f"n={n}") if args.workload == "dense" else
                                f"sparse exact Ryser (split-dd), n={n}, density 0.2, values U(0,1]"),
                   "n": n, "density": DENSITY if args.workload == "dense" else 0.2,
                   "values": "U{1,2,3,4}" if args.workload == "dense" else "U(0,1]",
                   "gray_steps_per_permanent": total_steps,
                   "parallelism": (f"{world} ranks: Gray-range shards of one matrix, 16-byte NCCL all-gather"
                                   if world > 1 else "1 rank, the whole walk"),
                   "l2": "256 MB buffer written between steps (operand is 12.8 KB; compute-bound)",
                   "timing": "CUDA events around each shard kernel (engine stream) and the all-gather; "
                             "max over ranks"},
        "result": {"permanent": perm_value, "matrix_seed": SEED},
        "e2e": {"value": args.steps * total_steps / e2e_s, "unit": "steps/s",
                "h2d_bytes_per_step": int(4 * n * n) * world, "d2h_bytes_per_step": 16 * world,
                "ms_per_step": e2e_s * 1e3 / args.steps, "path": e2e_path, "launches_per_call": 1},
        "e2e_with_accuracy_policy": policy,
        "roofline": {"bound": "fp64", "achieved": achieved / 1e12, "peak": peak_ops / 1e12, "unit": "TFLOP/s",
                     "frac": achieved / peak_ops, "traffic": traffic,
                     "peak_source": "measured this run: perm_fp64_peak (independent DFMA chains), "
                                    "1 op = 1 lane DADD/DMUL/DFMA",
                     "algorithmic": ops_text},
        "gpu_launches": args.steps * 1 + args.steps * 1,
        "wall_s_timed": wall,
    }
    if weak:
        line["weak_scaling"] = weak
    line["clocks"] = clk.summary()
    if kname in ("int32x", "tc", "int32x_dd"):
        # The integer and tensor-core kernels do not run the FP64-X algorithm:
        # their binding resource is instruction issue (one warp instruction per
        # cycle per SM sub-partition).  achieved = the kernel's warp
        # instructions per launch (ncu, profiles/) / the CUDA-event launch time;
        # peak = 4 x SMs x the median SM clock sampled during the timed region.
        fp64_equiv = line["roofline"]
        fp64_equiv["note"] = ("FP64-X-equivalent rate: this kernel moves the x updates off the FP64 pipe, "
                              "so it can exceed the FP64 roofline")
        sm_mhz = line["clocks"].get("sm_mhz") or 1965.0
        sms = torch.cuda.get_device_properties(device).multi_processor_count
        peak_issue = 4.0 * sms * sm_mhz * 1e6
        inst = prof_rec.get("warp_inst_per_launch") if prof_rec else None
        if inst and world > 1:
            inst = inst / world  # a shard walks 1/world of the Gray range
        ach = inst / (mean_ms * 1e-3) if inst else None
        line["roofline"] = {"bound": "issue", "achieved": ach / 1e12 if ach else None,
                            "peak": peak_issue / 1e12, "unit": "Twarp-inst/s",
                            "frac": ach / peak_issue if ach else None, "traffic": traffic,
                            "peak_source": f"4 warp instructions / cycle / SM x {sms} SMs x "
                                           f"{sm_mhz:.0f} MHz (median sampled SM clock)",
                            "algorithmic": "smsp__inst_executed.sum of one launch of "
                                           f"{kernel_template(kname, A)} (ncu, profiles/ryser_dense_n40_issue.json)",
                            "fp64_equivalent": fp64_equiv}
        if prof_stale:
            line["roofline"]["frac_stale"] = True
            line["roofline"]["stale_reason"] = prof_stale
    line["config"]["kernel"] = {1: "FP64-X register kernel", 3: "int32-X register kernel",
                                5: "tensor-core row sums (tcgen05 kind::i8) + int32 products",
                                7: "int32-X register kernel, double-double products and sum"}.get(r.kernel, r.kernel)
    if r.kernel == pb.PERM_KERNEL_DENSE_INT:
        line["config"]["kernel_instance"] = kernel_template("int32x", A)
    if rank == 0 and not args.no_secondary:
        line["secondary"] = secondary(pb, eng)
        # the same n=40 matrix through the int32-X and tensor-core kernels
        for key, v in (("dense_n40_int32x_same_matrix", pb.PERM_KERNEL_DENSE_INT),
                       ("dense_n40_tensor_core_same_matrix", pb.PERM_KERNEL_DENSE_TC)):
            rm = eng.upload_dense(A, variant=v)
            rm.run()
            ir = rm.run()
            rm.free()
            line["secondary"][key] = {"kernel_ms": ir.kernel_ms, "steps_per_s": total_steps / (ir.kernel_ms * 1e-3),
                                      "rel_diff_vs_headline": abs(ir.value - perm_value) / abs(perm_value)}
        # the same n=40 matrix through the FP64-X kernel (the kernel used for real-valued inputs)
        f64 = eng.upload_dense(A, variant=pb.PERM_KERNEL_DENSE)
        f64.run()
        fr = f64.run()
        f64.free()
        # FP64 operations the walk executes per Gray step: n updates and n - 1
        # multiplies (one level); in the two-level layout R inner rows at
        # seven of eight steps (R updates, R - 1 multiplies, times P_out); in
        # the three-level layout 2 R1 at four steps in eight, 2 R2 at three
        r1, r2l = pb.fp64_levels(A)
        if r1:
            executed = (4 * 2 * r1 + 3 * 2 * r2l + 2 * n - 1) / 8
        else:
            executed = (7 * 2 * r2l + 2 * n - 1) / 8 if r2l else 2 * n - 1
        line["secondary"]["dense_n40_fp64x_same_matrix"] = {
            "kernel_ms": fr.kernel_ms, "steps_per_s": total_steps / (fr.kernel_ms * 1e-3),
            "levels": [r1, r2l],
            "fp64_equivalent_frac_of_measured_peak": total_steps * ops_per_step / (fr.kernel_ms * 1e-3) / peak_ops,
            "fp64_pipe_frac_of_measured_peak": total_steps * executed / (fr.kernel_ms * 1e-3) / peak_ops,
            "rel_diff_vs_headline": abs(fr.value - perm_value) / abs(perm_value)}
        line["secondary"]["reference_gpu_same_box"] = reference_gpu(
            A, mean_ms, line["secondary"]["sparse_n36_d020_real"].get("auto_kernel_ms"),
            policy["value"] if policy else None)
        line["secondary"]["batched_8192_n12_28"] = batched_secondary(pb, eng)
        line["secondary"]["serving_poisson_2000_per_s"] = serving_secondary(pb, baseline=True)
        line["secondary"]["serving_poisson_40_per_s"] = serving_secondary(pb, requests=120, rate=40.0)
    if rank == 0 and not args.no_cpu_baseline:
        try:
            threads = os.cpu_count() or 1
            rate, steps, dt = cpu_reference_rate(A, 15.0, threads)
            line["cpu_baseline"] = {"value": rate, "unit": "steps/s", "cores": threads, "kind": "reference",
                                    "sample": f"Gray indices [1, {1 + steps}) of the same n=40 matrix "
                                              f"({dt:.1f} s), cpu_perman64 (gpu_exact_dense.cu:7)"}
        except Exception as e:
            line["cpu_baseline"] = {"value": None, "unavailable": str(e)}
    res.free()
    plain.close()
    eng.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank == 0:
        print(json.dumps(line))
    return 0


class _Capture:
    """Capture fd 1 (the reference's wrappers print their own kernel time,
    `kernel in <seconds>`, gpu_exact_dense.cu:679-683)."""

    def __enter__(self):
        import tempfile

        sys.stdout.flush()
        self.saved = os.dup(1)
        self.tmp = tempfile.TemporaryFile(mode="w+")
        os.dup2(self.tmp.fileno(), 1)
        return self

    def __exit__(self, *exc):
        sys.stdout.flush()
        os.dup2(self.saved, 1)
        os.close(self.saved)
        self.tmp.seek(0)
        self.text = self.tmp.read()
        self.tmp.close()

    def kernel_seconds(self):
        import re

        m = re.findall(r"kernel in ([0-9.eE+-]+)", getattr(self, "text", ""))
        return float(m[-1]) if m else None


def cfg2_matrix(n: int = 36):
    """The sparse exact configuration: n=36, Bernoulli(0.20) mask with no empty
    row or column, values U(0,1], seed 2026 (tests/golden holds its
    double-double value); other orders from the same generator."""
    rng = np.random.default_rng(2026)
    while True:
        mk = rng.random((n, n)) < 0.2
        if mk.any(0).all() and mk.any(1).all():
            break
    return mk * (1.0 - rng.random((n, n)))


def golden_value(name: str):
    try:
        data = json.loads((ROOT / "tests" / "golden" / "golden.json").read_text())
        for c in data["cases"]:
            if c["name"] == name:
                return c["dd"][0] + c["dd"][1]
    except Exception:
        pass
    return None


def reference_gpu(A40, ours_n40_ms, ours_cfg2_ms, certified_n40):
    """The reference's own GPU kernels (built for sm_100a from its sources) on
    the same box, kernel against kernel: its wrappers time the kernel alone
    (launch to cudaDeviceSynchronize, host clock, after a warm-up call that
    creates the context) and print it; allocation and copies are outside.
    -p4 (gpu_exact_dense.cu:641) on the headline n=40 matrix and -s -p7
    (gpu_exact_sparse.cu:1124, skipOrder) on the sparse configuration, each
    with its error against our certified value / the double-double oracle."""
    try:
        sys.path.insert(0, str(ROOT / "oracle"))
        from oracle import Reference

        ref = Reference()
        out = {}
        # warm-up: context creation and module load on a small matrix
        W = np.ascontiguousarray(np.ones((20, 20)), dtype=np.int32)
        with _Capture():
            ref.lib.ref_gpu_dense_mshared_i32(W.ctypes.data_as(ctypes.c_void_p), 20, 2048, 256)
        Mi = np.ascontiguousarray(A40, dtype=np.int32)
        with _Capture() as cap:
            t = time.perf_counter()
            v = ref.lib.ref_gpu_dense_mshared_i32(Mi.ctypes.data_as(ctypes.c_void_p), Mi.shape[0], 2048, 256)
            wall = time.perf_counter() - t
        ks = cap.kernel_seconds()
        steps = 2.0 ** (Mi.shape[0] - 1)
        out["p4_dense_n40_headline"] = {
            "kernel_s": ks, "wall_s_incl_alloc_copy": wall, "steps_per_s": steps / ks if ks else None,
            "value": v, "rel_error_vs_certified": abs(v - certified_n40) / abs(certified_n40) if certified_n40 else None,
            "ours_kernel_s": ours_n40_ms * 1e-3,
            "ours_speedup_kernel_vs_kernel": ks / (ours_n40_ms * 1e-3) if ks else None}
        B = cfg2_matrix()
        c = compress_for_reference(B)
        want = golden_value("cfg2_sparse_real_n36_d020")
        with _Capture() as cap:
            t = time.perf_counter()
            v = ref.lib.ref_gpu_skipper_f64(*c, 36, 2048, 128)
            wall = time.perf_counter() - t
        ks = cap.kernel_seconds()
        out["p7_skipper_cfg2_n36_d020"] = {
            "kernel_s": ks, "wall_s_incl_alloc_copy": wall, "dense_equivalent_steps_per_s": 2.0 ** 35 / ks if ks else None,
            "value": v, "rel_error_vs_dd_oracle": abs(v - want) / abs(want) if want else None,
            "ours_kernel_s": ours_cfg2_ms * 1e-3 if ours_cfg2_ms else None,
            "ours_speedup_kernel_vs_kernel": ks / (ours_cfg2_ms * 1e-3) if ks and ours_cfg2_ms else None}
        out["cuda_status_after"] = ref.lib.ref_last_cuda_error().decode()
        # its Monte-Carlo kernels (gpu_approximation_dense.cu:374, :528) on the
        # n=64 binary matrix of the mc_n64 secondary, 2e5 trials each, one call
        rng = np.random.default_rng(55)
        C = np.ascontiguousarray((rng.random((64, 64)) < 0.5).astype(np.float64))
        mc = {}
        with _Capture():
            t = time.perf_counter()
            v = ref.lib.ref_gpu_rasmussen_f64(C.ctypes.data_as(ctypes.c_void_p), 64, 200000)
            mc["rasmussen_seconds_incl_alloc_copy"] = time.perf_counter() - t
            mc["rasmussen_mean"] = v
            mc["rasmussen_cuda_status"] = ref.lib.ref_last_cuda_error().decode()
            t = time.perf_counter()
            v = ref.lib.ref_gpu_approximation_f64(C.ctypes.data_as(ctypes.c_void_p), 64, 200000, 4, 5)
            mc["scaling_seconds_incl_alloc_copy"] = time.perf_counter() - t
            mc["scaling_mean"] = v
            mc["scaling_cuda_status"] = ref.lib.ref_last_cuda_error().decode()
        out["mc_n64_binary_2e5_trials"] = mc
        return out
    except Exception as e:  # reported, never fatal
        return {"unavailable": str(e)}


def compress_for_reference(B):
    """skipOrder CRS/CCS (util.h:622) of B as the reference's SkipPer wrapper
    takes them: (mat, rptrs, cols, cptrs, rows, cvals) pointers, arrays kept
    alive on the function object."""
    pb = sys.modules["perman_b200"]
    c = pb.compress(2, B)
    arrs = [np.ascontiguousarray(c["mat"], dtype=np.float64), np.ascontiguousarray(c["rptrs"], dtype=np.int32),
            np.ascontiguousarray(c["cols"], dtype=np.int32), np.ascontiguousarray(c["cptrs"], dtype=np.int32),
            np.ascontiguousarray(c["rows"], dtype=np.int32), np.ascontiguousarray(c["cvals"], dtype=np.float64)]
    compress_for_reference.keep = arrs
    return [a.ctypes.data_as(ctypes.c_void_p) for a in arrs]


def batched_secondary(pb, eng, count=8192):
    """8192 matrices, n ~ U[12,28], density ~ U[0.2,0.9], half binary and half
    U(0,1], dense or sparse layout chosen per matrix by the batch: one
    persistent launch per captured graph, lane ranges and kernel variant from
    the autotuner; the comparison point is one launch per matrix of the plain
    kernel."""
    rng = np.random.default_rng(4444)
    mats = []
    for i in range(count):
        n = int(rng.integers(12, 29))
        d = rng.uniform(0.2, 0.9)
        while True:
            m = (rng.random((n, n)) < d).astype(np.float64)
            if m.any(0).all() and m.any(1).all():
                break
        if i % 2:
            m *= 1.0 - rng.random((n, n))
        mats.append(m)
    t = time.perf_counter()
    table = eng.batch_autotune(12, 28)
    tune_s = time.perf_counter() - t
    variant = eng.batch_variant()
    sparse_layout = sum(1 for m in mats if m.shape[0] >= 12 and pb.sdd_layout(m) > 0)
    t = time.perf_counter()
    b = eng.batch(mats)
    create_ms = (time.perf_counter() - t) * 1e3  # host layout choice and images, upload, graph capture
    t = time.perf_counter()
    eng.batch(mats).free()  # the same again, with the release of its device and pinned memory
    create_again_ms = (time.perf_counter() - t) * 1e3
    b.run()
    times = []
    for _ in range(3):
        vals, ms = b.run()
        times.append(ms)
    batch_ms = min(times)
    # the same replay plus the accuracy policy (exact zeros, cross-checks,
    # double-double) for matrices whose worst-case bound exceeds 1e-10
    pvals, est, reevaluated, policy_ms = b.run_ex()
    b.free()
    finite = est[np.isfinite(est)]
    # where the batch's time goes: the same replay on sub-batches (binary /
    # real, by order band), each timed alone; FP64-X-equivalent rate of the
    # real ones (2n FP64 ops per Gray step) against the live FP64 peak
    peak_ops = max(eng.fp64_peak()[0], eng.fp64_peak()[0])
    breakdown = {}
    kinds = ["binary" if i % 2 == 0 else "real" for i in range(count)]
    for kind in ("binary", "real"):
        for lo, hi in ((12, 20), (21, 24), (25, 26), (27, 28)):
            sel = [m for m, k in zip(mats, kinds) if k == kind and lo <= m.shape[0] <= hi]
            if not sel:
                continue
            sb = eng.batch(sel)
            sb.run()
            sub_ms = min(sb.run()[1] for _ in range(2))
            sb.free()
            st = sum(2.0 ** (m.shape[0] - 1) for m in sel)
            ops = sum(2.0 ** (m.shape[0] - 1) * 2 * m.shape[0] for m in sel)
            breakdown[f"{kind}_n{lo}_{hi}"] = {
                "matrices": len(sel), "ms": sub_ms, "gray_steps": st, "steps_per_s": st / (sub_ms * 1e-3),
                "fp64_equivalent_frac_of_peak": ops / (sub_ms * 1e-3) / peak_ops}
    breakdown["sum_of_parts_ms"] = sum(v["ms"] for v in breakdown.values() if isinstance(v, dict))
    # one launch per matrix (plain kernel, FP64 X, host loop through the C ABI;
    # a context without error estimates, like the plain batch replay above)
    with pb.Engine(eng.device) as plain:
        plain.set_rel_target(-1.0)
        for m in mats[:64]:
            plain.exact_dense(m, variant=pb.PERM_KERNEL_DENSE)
        t = time.perf_counter()
        ref_vals = [plain.exact_dense(m, variant=pb.PERM_KERNEL_DENSE).value for m in mats]
        per_ms = (time.perf_counter() - t) * 1e3
    # binary matrices without a perfect matching have permanent 0: both kernels
    # return rounding noise there, so relative differences use |perm| >= 1e-3
    err = max(abs(a - b) / abs(b) for a, b in zip(vals, ref_vals) if abs(b) >= 1e-3)
    noise = max((abs(a - b) for a, b in zip(vals, ref_vals) if abs(b) < 1e-3), default=0.0)
    steps = sum(2.0 ** (m.shape[0] - 1) for m in mats)
    return {"matrices": count, "batch_ms": batch_ms, "batch_perms_per_s": count / (batch_ms * 1e-3),
            "batch_steps_per_s": steps / (batch_ms * 1e-3),
            "one_launch_per_matrix_ms": per_ms, "one_launch_per_matrix_perms_per_s": count / (per_ms * 1e-3),
            "speedup_vs_one_launch_per_matrix": per_ms / batch_ms, "max_rel_diff_vs_single": err,
            "max_abs_diff_where_perm_below_1e-3": noise,
            "with_accuracy_policy": {"ms": policy_ms, "perms_per_s": count / (policy_ms * 1e-3),
                                     "reevaluated": reevaluated, "exact_zeros": int(np.sum(pvals == 0.0)),
                                     "max_rel_error_estimate": float(np.max(finite)) if finite.size else None,
                                     "unbounded_estimates": int(est.size - finite.size)},
            "create_ms": create_ms, "create_again_ms": create_again_ms, "autotune_s": tune_s,
            "autotuned_lane_log2": table,
            "autotuned_kernel_variant": variant,
            "matrices_with_a_sparse_column_triple": sparse_layout, "breakdown": breakdown,
            "timing": "CUDA events around the graph launch (queue reset + kernel + 128 KB readback)"}


def serving_secondary(pb, requests=400, rate=2000.0, slots=4, seed=5555, baseline=False):
    """Poisson arrivals mixing exact (n ~ U[16,34], U(0,1], d=0.5) and
    approximate (binary n ~ U[40,64], d=0.5, Rasmussen or scaling y=4 z=5,
    2e5 trials) requests through the request loop; with `baseline`, the same
    requests also run one call at a time on one context (the same accuracy
    policy) for the one-launch-per-request comparison."""
    import threading

    rng = np.random.default_rng(seed)
    reqs = []
    for i in range(requests):
        if rng.random() < 0.5:
            n = int(rng.integers(16, 35))
            A = (rng.random((n, n)) < 0.5) * (1.0 - rng.random((n, n)))
            reqs.append((pb.PERM_REQ_EXACT_DENSE, A, {}))
        else:
            n = int(rng.integers(40, 65))
            A = (rng.random((n, n)) < 0.5).astype(np.float64)
            kind = pb.PERM_REQ_RASMUSSEN if rng.random() < 0.5 else pb.PERM_REQ_SCALING
            reqs.append((kind, A, {"trials": 200000, "scale_intervals": 4, "scale_times": 5, "seed": i}))
    gaps = rng.exponential(1.0 / rate, requests)
    with pb.Server(0, slots=slots) as srv:
        tickets = [None] * requests

        def feeder():
            t0 = time.perf_counter()
            due = 0.0
            for i, (k, A, kw) in enumerate(reqs):
                due += gaps[i]
                while time.perf_counter() - t0 < due:
                    time.sleep(min(0.0005, max(0.0, due - (time.perf_counter() - t0))))
                tickets[i] = srv.submit(k, A, **kw)

        th = threading.Thread(target=feeder)
        t0 = time.perf_counter()
        th.start()
        th.join()
        resps = [srv.wait(t) for t in tickets]
        wall = time.perf_counter() - t0
    lat = np.array([r["t_done_ms"] - r["t_submit_ms"] for r in resps])
    ok = sum(r["status"] == 0 for r in resps)
    errors = sorted({f'{r["status"]}: {r["message"]}' for r in resps if r["status"] != 0})[:5]
    first = min(r["t_submit_ms"] for r in resps)
    last = max(r["t_done_ms"] for r in resps)
    dev = sum(r["device_ms"] for r in resps)
    out = {"requests": requests, "offered_rate_per_s": rate, "slots": slots, "ok": ok,
           "perms_per_s": requests / ((last - first) * 1e-3), "p50_ms": float(np.percentile(lat, 50)),
           "p99_ms": float(np.percentile(lat, 99)), "mean_device_ms_per_request": dev / requests,
           "errors": errors,
           "wall_s": wall}
    if baseline:
        eng = pb.Engine(0)
        t0 = time.perf_counter()
        for k, A, kw in reqs:
            if k == pb.PERM_REQ_EXACT_DENSE:
                eng.exact_dense(A)
            elif k == pb.PERM_REQ_RASMUSSEN:
                eng.rasmussen(A, kw["trials"], seed=kw["seed"])
            else:
                eng.scaling(A, kw["trials"], 4, 5, seed=kw["seed"])
        seq = time.perf_counter() - t0
        eng.close()
        out["one_call_per_request"] = {"wall_s": seq, "perms_per_s": requests / seq,
                                       "served_speedup": (requests / ((last - first) * 1e-3)) / (requests / seq)}
    return out


def secondary(pb, eng):
    """The other exact workloads, timed once each (parity cases, not bench lines)."""
    out = {}
    rng = np.random.default_rng(101)
    while True:
        m = (rng.random((30, 30)) < 0.5).astype(np.float64)
        if m.any(0).all() and m.any(1).all():
            break
    r = eng.exact_dense(m)
    r = eng.exact_dense(m)
    out["dense_n30_binary"] = {"kernel_ms": r.kernel_ms, "steps_per_s": r.total_steps / (r.kernel_ms * 1e-3),
                               "permanent": r.value}
    rng = np.random.default_rng(2026)
    while True:
        mk = rng.random((36, 36)) < 0.2
        if mk.any(0).all() and mk.any(1).all():
            break
    B = mk * (1.0 - rng.random((36, 36)))
    c = pb.compress(2, B)
    s = eng.exact_sparse(c["n"], c["rptrs"], c["cols"], c["rvals"], c["cptrs"], c["rows"], c["cvals"],
                         variant=pb.PERM_KERNEL_SKIPPER)
    d = eng.exact_sparse(c["n"], c["rptrs"], c["cols"], c["rvals"], c["cptrs"], c["rows"], c["cvals"])
    out["sparse_n36_d020_real"] = {"skipper_kernel_ms": s.kernel_ms, "skipper_visited": s.steps,
                                   "dense_equivalent": s.total_steps,
                                   "skipper_steps_per_s": s.total_steps / (s.kernel_ms * 1e-3),
                                   "auto_kernel": d.kernel, "auto_kernel_ms": d.kernel_ms,
                                   "auto_steps_per_s": d.total_steps / (d.kernel_ms * 1e-3), "permanent": d.value,
                                   "rel_diff_skipper_vs_auto": abs(s.value - d.value) / abs(d.value)}
    # a sparse binary case where SkipPer skips most of the walk
    rng = np.random.default_rng(36)
    P = ((np.eye(36) + np.eye(36)[rng.permutation(36)] + np.eye(36)[rng.permutation(36)]) > 0).astype(np.float64)
    cp = pb.compress(2, P)
    sp = eng.exact_sparse(cp["n"], cp["rptrs"], cp["cols"], cp["rvals"], cp["cptrs"], cp["rows"], cp["cvals"],
                          variant=pb.PERM_KERNEL_SKIPPER)
    dp = eng.exact_dense(cp["mat"])
    out["sparse_n36_three_per_row_binary"] = {"skipper_kernel_ms": sp.kernel_ms, "skipper_visited": sp.steps,
                                              "dense_equivalent": sp.total_steps, "dense_kernel_ms": dp.kernel_ms,
                                              "permanent": sp.value}
    rng = np.random.default_rng(55)
    C = (rng.random((64, 64)) < 0.5).astype(np.float64)
    eng.rasmussen(C, 2000, seed=1)
    t = time.perf_counter()
    e = eng.rasmussen(C, 200000, seed=1)
    e_wall = time.perf_counter() - t
    t = time.perf_counter()
    f = eng.scaling(C, 200000, 4, 5, seed=2)
    f_wall = time.perf_counter() - t
    out["mc_n64_binary_2e5_trials"] = {"rasmussen_trials_per_s": 200000 / (e.kernel_ms * 1e-3),
                                       "scaling_trials_per_s": 200000 / (f.kernel_ms * 1e-3),
                                       "rasmussen_ms": e.kernel_ms, "rasmussen_call_s": e_wall,
                                       "rasmussen_mean": e.mean, "rasmussen_rel_se": e.std_error / e.mean,
                                       "scaling_ms": f.kernel_ms, "scaling_call_s": f_wall, "scaling_mean": f.mean,
                                       "scaling_rel_se": f.std_error / f.mean}
    # the accuracy policy on the request loop's real matrices (density 0.5,
    # U(0,1]): the kernel it plans from the device prediction of the FP64-X
    # bound, that prediction against the FP64-X walk's own bound, and the
    # policy's device time in FP64-X walks
    rng = np.random.default_rng(5555)
    pol = {}
    for n in (28, 30, 32, 34):
        A = (rng.random((n, n)) < 0.5) * (1.0 - rng.random((n, n)))
        kern, predicted = eng.dense_plan(A)
        f = eng.exact_dense(A, variant=pb.PERM_KERNEL_DENSE)
        eng.exact_dense(A)
        r = eng.exact_dense(A)
        pol[f"n{n}"] = {"planned_kernel": kern, "predicted_fp64_bound": predicted,
                        "fp64_walk_bound": f.rel_error_estimate, "fp64_walk_ms": f.kernel_ms,
                        "policy_kernel": r.kernel, "policy_ms": r.kernel_ms,
                        "split_dd_levels": list(pb.sdd_levels(A)),
                        "policy_in_fp64_walks": r.kernel_ms / f.kernel_ms,
                        "policy_rel_error_estimate": r.rel_error_estimate}
    out["policy_real_dense_d050"] = pol
    return out


if __name__ == "__main__":
    sys.exit(main())

#!/usr/bin/env python
"""bench.py — commit+fold elements/s at 2^22 F162 (suite l, Opening::Clear) on B200.

One step is one pass of the hot path over one witness: Prover::commit (3 limbs: 3889, 2917, 4861)
then Prover::fold with the round's folding challenges (crates/bench/src/bin/labinius.rs:104-130,
the `commit` and `fold` rows). `value` times the step on the device with the witness resident in
HBM; `e2e` times it through the public API with host buffers (pinned witness upload, commitment and
folded witness read back). Under torchrun every rank commits and folds its own witness (weak
scaling, no collective: witnesses are independent objects).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--config l]
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

MATRIX_SEED = bytes([0x5A]) * 32
WITNESS_SEED = bytes([0xC7]) * 32
DOMAIN = b"labinius/reference"
METRIC = "commit+fold elems/s at 2^22 (suite l, Clear, bit-exact)"
CONFIGS = {"s": 0, "m": 1, "l": 2, "xl": 3}


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="l", choices=list(CONFIGS))
    ap.add_argument("--cpu-seconds", type=float, default=15.0, help="budget of the CPU-baseline sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    return ap.parse_args()


def dist():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def init_group(world, backend):
    if world > 1:
        import datetime

        import torch.distributed as td

        os.environ.setdefault("MASTER_ADDR", "127.0.0.1")
        td.init_process_group(backend, timeout=datetime.timedelta(seconds=300))


def allreduce_max(x, world, device=None):
    if world == 1:
        return x
    import torch
    import torch.distributed as td

    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    td.all_reduce(t, op=td.ReduceOp.MAX)
    return float(t.item())


def barrier(world):
    if world > 1:
        import torch.distributed as td

        td.barrier()


# ------------------------------------------------------------------------------------------------
# clocks during the timed region
# ------------------------------------------------------------------------------------------------
class Clocks:
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={self.index}", f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except OSError:
            self.p = None

    def stop(self):
        if self.p is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.f.read().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.f.name)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


# ------------------------------------------------------------------------------------------------
# CPU baseline: the oracle (a scalar C++ restatement of the reference's algorithm) on a sample
# ------------------------------------------------------------------------------------------------
def cpu_baseline(params_tuple, budget_s, threads):
    """Time the oracle's commit on a sample of columns and its fold on a sample of ring elements,
    and scale each to the full round: elems/s = n / (t_commit_full + t_fold_full)."""
    import oracle as O

    O.build.build()
    wl, cl, primes = params_tuple
    P = O.Params(wl, cl, primes, 0)
    A = O.key_expand(P, O.key_seed(MATRIX_SEED))
    w = O.witness_random(P.witness_len, WITNESS_SEED)
    t = O.Transcript(DOMAIN)
    ch = np.zeros(P.columns, O.CHALLENGE_DTYPE)
    t.absorb_u64(1)
    for j in range(P.columns):
        ch[j] = O.sample_short_challenge(t)[0]
    # calibrate on one column / a few ring elements, then size the sample to the budget
    t0 = time.perf_counter()
    O.commit(P, A, w, 0, 1, threads=1)
    per_col = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.fold(P, w, ch, 0, 4, threads=1)
    per_ring = (time.perf_counter() - t0) / 4
    cols = max(threads, int(0.5 * budget_s * threads / max(per_col, 1e-9)) // threads * threads)
    cols = min(cols, P.columns)
    rings = max(threads, int(0.5 * budget_s * threads / max(per_ring, 1e-9)) // threads * threads)
    rings = min(rings, P.len_ring)
    t0 = time.perf_counter()
    O.commit(P, A, w, 0, cols, threads=threads)
    tc = time.perf_counter() - t0
    t0 = time.perf_counter()
    O.fold(P, w, ch, 0, rings, threads=threads)
    tf = time.perf_counter() - t0
    full = tc * P.columns / cols + tf * P.len_ring / rings
    return {"value": P.witness_len / full, "unit": "elems/s", "cores": threads, "kind": "port",
            "sample": f"oracle commit of {cols}/{P.columns} columns ({tc:.2f} s) and fold of {rings}/{P.len_ring} "
                      f"ring elements ({tf:.2f} s) at 2^{wl}, scaled to the full round; {threads} threads"}


def suite_shape(config):
    from labinius_b200 import SUITES, Opening, Params

    params = Params.sized(SUITES[CONFIGS[config]], Opening.clear())
    return params


# ------------------------------------------------------------------------------------------------
# the reference arm
# ------------------------------------------------------------------------------------------------
def run_reference(args):
    rank, world, local = dist()
    if rank != 0:
        return 0
    params = suite_shape(args.config)
    shape = (params.witness_log_len, params.column_log_len, params.primes())
    threads = os.cpu_count() or 1
    vals = []
    budget = max(2.0, min(args.cpu_seconds, 60.0 / max(1, args.steps + args.warmup)))
    for i in range(args.warmup + args.steps):
        r = cpu_baseline(shape, budget, threads)
        if i >= args.warmup:
            vals.append(r)
    value = float(np.median([v["value"] for v in vals]))
    line = {"metric": METRIC, "value": value, "unit": "elems/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1000.0 * params.witness_len() / value, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 mod q / GF(2)", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": f"suite {args.config}: 2^{params.witness_log_len} F162, {params.columns()} columns, "
                                   f"moduli {params.primes()}, Clear", "cpu_threads": threads},
            "cpu_baseline": {"value": value, "unit": "elems/s", "cores": threads, "kind": "port",
                             "sample": vals[-1]["sample"]},
            "e2e": {"value": value, "unit": "elems/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------
# our arm
# ------------------------------------------------------------------------------------------------
def run_ours(args):
    import ctypes

    import torch

    rank, world, local = dist()
    torch.cuda.set_device(local)
    init_group(world, "nccl")
    import labinius_b200 as L
    from labinius_b200._native import check, lib, ptr

    params = suite_shape(args.config)
    n, r = params.witness_len(), params.columns()
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    wseed = bytes([(0xC7 + rank) & 0xFF]) * 32
    w = L.Witness.random(pp, wseed)
    prover = L.Prover(pp)
    verifier = L.Verifier(pp)
    # the round's real folding challenges
    c0, op0 = prover.commit(w)
    t = L.Transcript(DOMAIN)
    point = verifier.derive_evaluation_point(t, c0)
    row = w.row_evaluate(point)
    ch = verifier.derive_folding_challenges(t, row)
    prover.recycle(op0)
    chal = np.ascontiguousarray(ch.challenges)
    N = lib()
    stream = torch.cuda.ExternalStream(N.lbg_prover_stream(prover._h))
    flush = torch.empty(64 * 1024 * 1024, dtype=torch.int32, device="cuda")  # 256 MB > 126 MB L2

    def step():
        op = ctypes.c_void_p()
        check(N.lbg_commit(prover._h, w._h, None, None, None, ctypes.byref(op)))
        check(N.lbg_fold(prover._h, op, ptr(chal), len(chal), None))

    for _ in range(args.warmup):
        step()
    check(N.lbg_prover_sync(prover._h))
    # row evaluation and mle, reported beside the metric
    tr0 = time.perf_counter()
    for _ in range(3):
        w.row_evaluate(point)
    t_row = (time.perf_counter() - tr0) / 3
    tm0 = time.perf_counter()
    for _ in range(3):
        w.mle_evaluate(point)
    t_mle = (time.perf_counter() - tm0) / 3

    check(N.lbg_prover_profile(prover._h, 1))
    launches0 = N.lbg_prover_launch_count(prover._h)
    clocks = Clocks(local)
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clocks.start()
    evs = []
    for _ in range(args.steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(stream)
        step()
        b.record(stream)
        evs.append((a, b))
    check(N.lbg_prover_sync(prover._h))
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = sum(a.elapsed_time(b) for a, b in evs) / args.steps
    launches = int(N.lbg_prover_launch_count(prover._h) - launches0)
    ms_max = allreduce_max(ms, world, "cuda")
    value = world * n / (ms_max / 1000.0)

    stats = {}
    for name in ["commit", "commit_finish", "challenge_slots", "fold"]:
        cnt, tot = ctypes.c_uint64(), ctypes.c_double()
        check(N.lbg_prover_kernel_stats(prover._h, name.encode(), ctypes.byref(cnt), ctypes.byref(tot)))
        stats[name] = (int(cnt.value), float(tot.value))
    check(N.lbg_prover_profile(prover._h, 0))

    # roofline of the dominant kernel (commit, one launch per limb): algorithmic bytes per launch =
    # the witness (24 B per F162) + the key's component form (32 B per ring element and leaf) + the
    # limb's commitment (16 B per column and leaf)
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except (OSError, ValueError):
        pass
    hbm = float(peaks.get("hbm_gbs", 6650.0))
    peak_src = "measured" if "hbm_gbs" in peaks else "fallback"
    cnt, tot = stats["commit"]
    per_launch_ms = tot / max(cnt, 1)
    len_ring = params.len_ring()
    algo_bytes = 24 * n + len_ring * 162 * 32 + r * 162 * 16
    achieved = algo_bytes / (per_launch_ms / 1000.0) / 1e9
    traffic = None
    try:
        traffic = json.load(open(os.path.join(ROOT, "profiles", "traffic.json"))).get(f"commit_{args.config}")
    except (OSError, ValueError):
        pass
    # integer-pipe view: 32-bit integer ops per F162 per limb of the commit kernel (the 162-point
    # transform: 54 radix-3 butterflies x 3 levels x 15 ops + 27 window lookups + 162 reductions x 3;
    # the module multiply-accumulate: 648 multiply-adds)
    int_ops = n * (162 * 15 + 27 * 8 + 162 * 3 + 648)
    fold_ms = stats["fold"][1] / max(stats["fold"][0], 1)

    e2e = None
    if not args.no_e2e:
        host_w = torch.empty((n, 3), dtype=torch.int64, pin_memory=True)
        hw = host_w.numpy().view(np.uint64)
        hw[:] = w.elements()
        L_ = len(params.primes())
        mat = torch.empty((r, 4, L_, 162), dtype=torch.int16, pin_memory=True).numpy()
        vout = torch.empty((params.len_ring(), 648), dtype=torch.int16, pin_memory=True).numpy()

        def e2e_step():
            wh = ctypes.c_void_p()
            check(N.lbg_witness_from_host(pp._h, ptr(hw), n, ctypes.byref(wh)))
            op = ctypes.c_void_p()
            check(N.lbg_commit(prover._h, wh, ptr(mat), None, None, ctypes.byref(op)))
            check(N.lbg_fold(prover._h, op, ptr(chal), len(chal), ptr(vout)))
            N.lbg_witness_free(wh)

        for _ in range(2):
            e2e_step()
        torch.cuda.synchronize()
        barrier(world)
        t0 = time.perf_counter()
        for _ in range(args.steps):
            e2e_step()
        torch.cuda.synchronize()
        e2e_ms = allreduce_max((time.perf_counter() - t0) * 1000.0 / args.steps, world, "cuda")
        e2e = {"value": world * n / (e2e_ms / 1000.0), "unit": "elems/s", "ms_per_step": e2e_ms,
               "h2d_bytes_per_step": 24 * n + chal.nbytes, "d2h_bytes_per_step": mat.nbytes + vout.nbytes,
               "timing": "host wall clock around synchronous API calls, max over ranks"}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline((params.witness_log_len, params.column_log_len, params.primes()), args.cpu_seconds,
                           os.cpu_count() or 1)

    line = {
        "metric": METRIC, "value": value, "unit": "elems/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 mod q / GF(2)", "data": "synthetic",
        "config": {"workload": f"suite {args.config}: 2^{params.witness_log_len} F162 in {r} columns, moduli "
                               f"{params.primes()}, Opening::Clear, Witness::random(seed)",
                   "l2": "flushed (256 MB write) before every timed step", "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": peak_src, "traffic": traffic, "kernel": "k_commit (one launch per limb)",
                     "per_launch_ms": per_launch_ms, "algorithmic_bytes_per_launch": algo_bytes,
                     "int_pipe": {"ops_per_launch": int_ops, "achieved_tops": int_ops / (per_launch_ms / 1000) / 1e12,
                                  "note": "integer-pipe bound; ops counted from the kernel's arithmetic"}},
        "kernels_ms": {k: {"launches": c, "avg_ms": (tt / c if c else None)} for k, (c, tt) in stats.items()},
        "t_commit_ms": stats["commit"][1] / args.steps + stats["commit_finish"][1] / args.steps,
        "t_fold_ms": (stats["fold"][1] + stats["challenge_slots"][1]) / args.steps,
        "t_fold_kernel_ms": fold_ms,
        "t_row_evaluate_ms": t_row * 1000, "t_mle_ms": t_mle * 1000,
        "gpu_launches": launches,
        "clocks": clk,
        "cpu_baseline": cpu,
        "e2e": e2e,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    del prover, w, pp
    if world > 1:
        import torch.distributed as td

        td.destroy_process_group()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

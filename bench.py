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
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--batch-instances", type=int, default=64)
    ap.add_argument("--no-served", action="store_true")
    ap.add_argument("--no-switch", action="store_true")
    ap.add_argument("--no-wire", action="store_true")
    ap.add_argument("--switch-sizes", default="18,20,22", help="log2 trace lengths of the switch line")
    ap.add_argument("--no-ntt", action="store_true")
    ap.add_argument("--no-suites", action="store_true")
    ap.add_argument("--ntt-count", type=int, default=1 << 20, help="ring elements of the NTT microbenchmark")
    ap.add_argument("--served-requests", type=int, default=10000)
    ap.add_argument("--served-plain-sample", type=int, default=200)
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


def rank_witness_seed(rank):
    """Rank r's own witness: the bench's seed [0xC7; 32] moved by r, so ranks commit different
    witnesses (weak scaling over independent objects)."""
    return bytes([(0xC7 + rank) & 0xFF]) * 32


def whole_job_value(world, n, ms_max):
    """Elements per second of the whole job: every rank's n elements over the slowest rank's time."""
    return world * n / (ms_max / 1000.0)


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
# CPU baseline: the oracle (a scalar C++ restatement of the reference's algorithm), whole steps
# ------------------------------------------------------------------------------------------------
class OracleStep:
    """The bench's step on the oracle: commit of every column on every limb, then the fold of every
    ring element with the round's folding challenges (crates/bench/src/bin/labinius.rs:104-130, the
    `commit` and `fold` rows). The challenges come from the oracle's own round (evaluation point,
    row evaluation, FoldingChallenges::derive) on its first commitment, outside any timed step."""

    def __init__(self, params_tuple, witness_seed=None):
        import oracle as O

        O.build.build()
        self.O = O
        wl, cl, primes = params_tuple
        self.P = O.Params(wl, cl, primes, 0)
        self.A = O.key_expand(self.P, O.key_seed(MATRIX_SEED))
        self.w = O.witness_random(self.P.witness_len, witness_seed or WITNESS_SEED)
        self.ch = None

    def challenges(self, C):
        O = self.O
        t = O.Transcript(DOMAIN)
        p0, _ = O.derive_evaluation_point(self.P, MATRIX_SEED, t, C=C)
        u = O.row_evaluate(self.w, p0)
        self.ch = O.derive_folding_challenges(self.P, t, u)
        return self.ch

    def step(self, threads, ch=None):
        """One whole step; returns (C, v, commit seconds, fold seconds)."""
        O = self.O
        t0 = time.perf_counter()
        C = O.commit(self.P, self.A, self.w, threads=threads)
        tc = time.perf_counter() - t0
        if ch is None:
            ch = self.ch if self.ch is not None else self.challenges(C)
        t0 = time.perf_counter()
        v = O.fold(self.P, self.w, ch, threads=threads)
        tf = time.perf_counter() - t0
        return C, v, tc, tf

    def single_thread(self):
        """The oracle on one thread: one column's commit and four ring elements' fold, scaled to
        the whole step (a sample: a full one-thread step takes minutes)."""
        O = self.O
        ch = self.ch if self.ch is not None else np.zeros(self.P.columns, O.CHALLENGE_DTYPE)
        t0 = time.perf_counter()
        O.commit(self.P, self.A, self.w, 0, 1, threads=1)
        tc = time.perf_counter() - t0
        t0 = time.perf_counter()
        O.fold(self.P, self.w, ch, 0, 4, threads=1)
        tf = time.perf_counter() - t0
        full = tc * self.P.columns + tf * self.P.len_ring / 4
        return {"value": self.P.witness_len / full, "unit": "elems/s", "cores": 1, "kind": "port",
                "sample": f"oracle commit of 1/{self.P.columns} columns ({tc:.3f} s) and fold of "
                          f"4/{self.P.len_ring} ring elements ({tf:.3f} s) on one thread, scaled to the step"}


def host_cpu():
    """The host's CPU model, for the baseline's record."""
    try:
        for line in open("/proc/cpuinfo"):
            if line.startswith("model name"):
                return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def cpu_baseline(params_tuple, threads, ch):
    """One whole oracle step on all host threads with the GPU round's challenges; returns the
    baseline record and the oracle's commitment and folded witness (the bench's parity check)."""
    s = OracleStep(params_tuple)
    C, v, tc, tf = s.step(threads, ch)
    s.ch = ch
    rec = {"value": s.P.witness_len / (tc + tf), "unit": "elems/s", "cores": threads, "kind": "port",
           "sample": f"one whole step: oracle commit of {s.P.columns}/{s.P.columns} columns ({tc:.2f} s) and "
                     f"fold of {s.P.len_ring}/{s.P.len_ring} ring elements ({tf:.2f} s) at 2^{s.P.witness_log_len}; "
                     f"{threads} threads, unpinned, on {host_cpu()}",
           "single_thread": s.single_thread()}
    return rec, C, v


def suite_shape(config):
    from labinius_b200 import SUITES, Opening, Params

    params = Params.sized(SUITES[CONFIGS[config]], Opening.clear())
    return params


def bench_config(config, params, world):
    """The `config` of both arms' lines (the same dict, so the lines compare)."""
    return {"workload": f"suite {config}: 2^{params.witness_log_len} F162 in {params.columns()} columns, moduli "
                        f"{params.primes()}, Opening::Clear, Witness::random(seed)",
            "l2": "flushed (256 MB write) before every timed step", "parallelism": f"replicas x{world}"}


# ------------------------------------------------------------------------------------------------
# the reference arm
# ------------------------------------------------------------------------------------------------
def run_reference(args):
    """The reference's algorithm on the host cores: the oracle port (the reference is a Rust
    workspace and no Rust toolchain exists here or on the GPU box), whole steps of the bench's
    workload on every host thread, timed by the host clock; warm-up steps untimed."""
    rank, world, local = dist()
    if rank != 0:
        return 0
    params = suite_shape(args.config)
    threads = os.cpu_count() or 1
    s = OracleStep((params.witness_log_len, params.column_log_len, params.primes()))
    for _ in range(args.warmup):
        s.step(threads)
    times = []
    for _ in range(args.steps):
        _, _, tc, tf = s.step(threads)
        times.append(tc + tf)
    ms = 1000.0 * sum(times) / len(times)
    value = params.witness_len() / (ms / 1000.0)
    line = {"metric": METRIC, "value": value, "unit": "elems/s", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "u32 mod q / GF(2)", "data": "synthetic",
            "impl": "reference",
            "config": bench_config(args.config, params, world),
            "cpu_baseline": {"value": value, "unit": "elems/s", "cores": threads, "kind": "port",
                             "sample": f"{args.steps} whole steps (commit of all {params.columns()} columns on "
                                       f"{len(params.primes())} limbs + fold of all {params.len_ring()} ring "
                                       f"elements), {threads} threads, unpinned, on {host_cpu()}",
                             "single_thread": s.single_thread()},
            "e2e": {"value": value, "unit": "elems/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)
    return 0


# ------------------------------------------------------------------------------------------------
# batched: 64 uneven witnesses under one key, against 64 sequential single-instance calls
# ------------------------------------------------------------------------------------------------
def run_batched(instances, steps, flush_bytes=256 << 20):
    """Sizes log2 n ~ U[16, 22] (seeded, rounded), each instance Params(log n, max(1, log n - 11),
    [3889, 9721]): column length 2048 F162 for all, so one key serves every instance. A step is the
    batched commit + fold of all instances (graphs on, schedule autotuned), timed with CUDA events on
    the batch's stream; the comparison is the same work as one single-instance commit + fold per
    instance (device time summed over the calls, and wall clock around the loop)."""
    import ctypes

    import torch

    import labinius_b200 as L
    from labinius_b200._native import check, lib, ptr
    from labinius_b200.batch import Batch

    rng = np.random.default_rng(2026)
    logs = np.rint(rng.uniform(16, 22, instances)).astype(int)
    col_logs = [max(1, int(l) - 11) for l in logs]
    seeds = [bytes([(0x21 + 7 * i) & 0xFF, i & 0xFF]) * 16 for i in range(instances)]
    total = int(sum(1 << (11 + c) for c in col_logs))
    pp = L.PublicParameters.from_seed(L.Params.new(11 + col_logs[0], col_logs[0], [L.Modulus.Q9721_FS_S]), MATRIX_SEED)
    b = Batch(pp, col_logs)
    b.witness_random(seeds)
    tuned = b.autotune()
    b.use_graphs(True)
    rounds = b.round(DOMAIN)
    chs = [r.challenges for r in rounds]
    stream = torch.cuda.ExternalStream(b.stream())
    flush = torch.empty(flush_bytes // 4, dtype=torch.int32, device="cuda")
    for _ in range(2):
        b.commit_device()
        b.fold(chs, read_back=False)
    torch.cuda.synchronize()
    l0 = b.launch_count()
    ms = 0.0
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        b.commit_device()
        b.fold(chs, read_back=False)
        e1.record(stream)
        e1.synchronize()
        ms += e0.elapsed_time(e1)
    ms /= steps
    launches = (b.launch_count() - l0) // steps

    # the same instances one by one through the single-instance path
    pps, provers, wits = {}, {}, []
    for i, c in enumerate(col_logs):
        if c not in pps:
            pps[c] = L.PublicParameters.from_seed(L.Params.new(11 + c, c, [L.Modulus.Q9721_FS_S]), MATRIX_SEED)
            provers[c] = L.Prover(pps[c])
        wits.append(L.Witness.random(pps[c], seeds[i]))
    N = lib()
    chal = [np.ascontiguousarray(ch) for ch in chs]

    def one(i):
        c = col_logs[i]
        op = ctypes.c_void_p()
        check(N.lbg_commit(provers[c]._h, wits[i]._h, None, None, None, ctypes.byref(op)))
        check(N.lbg_fold(provers[c]._h, op, ptr(chal[i]), len(chal[i]), None))

    for i in range(instances):
        one(i)
    torch.cuda.synchronize()
    seq_dev, seq_wall = 0.0, 0.0
    by_size = {}  # log2 n -> [instances, device ms summed over the steps]
    for _ in range(steps):
        with torch.cuda.stream(stream):
            flush.zero_()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for i in range(instances):
            c = col_logs[i]
            st = torch.cuda.ExternalStream(N.lbg_prover_stream(provers[c]._h))
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(st)
            one(i)
            e1.record(st)
            e1.synchronize()
            dt = e0.elapsed_time(e1)
            seq_dev += dt
            bs = by_size.setdefault(int(logs[i]), [0, 0.0])
            bs[0] += 1
            bs[1] += dt
        seq_wall += (time.perf_counter() - t0) * 1000
    seq_dev /= steps
    seq_wall /= steps
    # per size: the single-instance path's device rate. Batching runs the same per-element work, so
    # its device time is at best the elements at the best single-instance rate: that bounds the ratio.
    per_size = {str(lg): {"instances": v[0] // steps, "device_ms_each": v[1] / v[0],
                          "elems_s": (1 << lg) / (v[1] / v[0] / 1000)} for lg, v in sorted(by_size.items())}
    best_rate = max(v["elems_s"] for v in per_size.values())
    ceiling = seq_dev / (total / best_rate * 1000)

    # the whole round (commit, evaluation point, mle and row evaluation, folding challenges, fold):
    # the batch's device round (one graph, transcripts on the device, results read back) against one
    # plain API round per instance, both by the host clock around the calls
    b.round(DOMAIN, copy=False)
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for _ in range(steps):
        b.round(DOMAIN, copy=False)  # results read back into the batch's page-locked buffers
    round_ms = (time.perf_counter() - t0) * 1000 / steps
    verifiers = {c: L.Verifier(pps[c]) for c in pps}

    def plain_round(i):
        c = col_logs[i]
        cm, op = provers[c].commit(wits[i])
        t = L.Transcript(DOMAIN)
        point = verifiers[c].derive_evaluation_point(t, cm)
        wits[i].mle_evaluate(point)
        row = wits[i].row_evaluate(point)
        ch = verifiers[c].derive_folding_challenges(t, row)
        provers[c].fold(op, ch)

    plain_round(0)
    t0 = time.perf_counter()
    for i in range(instances):
        plain_round(i)
    plain_round_ms = (time.perf_counter() - t0) * 1000
    return {"value": total / (ms / 1000), "unit": "elems/s", "ms_per_step": ms, "instances": instances,
            "elements": total, "log2_sizes": [int(x) for x in logs],
            "sequential_device_ms": seq_dev, "sequential_wall_ms": seq_wall,
            "speedup_vs_sequential_device": seq_dev / ms, "speedup_vs_sequential_wall": seq_wall / ms,
            "sequential_by_log2_n": per_size, "ceiling_vs_sequential_device": ceiling,
            "schedule": tuned, "gpu_launches_per_step": launches, "graphs": True,
            "workload": "commit (2 limbs: 3889, 9721) + fold of every instance, column length 2048",
            "round": {"batched_ms": round_ms, "sequential_plain_ms": plain_round_ms,
                      "batched_elems_s": total / (round_ms / 1000), "sequential_plain_elems_s": total / (plain_round_ms / 1000),
                      "speedup": plain_round_ms / round_ms,
                      "workload": "commit + open of every instance: the batch's device round (graph, device "
                                  "transcripts, outputs read back) vs one plain API round per instance"}}


def run_suites(steps, flush_bytes=256 << 20):
    """Every size suite of Params::sized (crates/pcs/src/scheme/params.rs:91-128) in Opening::Clear
    and bit-dropped mode, plain single-instance path: commit + fold on the device (L2 flushed
    before each step, CUDA events on the prover's stream, the round's real folding challenges),
    plus Params::basic() (suite s) as a whole round through the public API and as the device round."""
    import ctypes

    import torch

    import labinius_b200 as L
    from labinius_b200._native import check, lib, ptr
    from labinius_b200.batch import Batch

    N = lib()
    flush = torch.empty(flush_bytes // 4, dtype=torch.int32, device="cuda")
    out = []
    for suite in L.SUITES:
        for opening in (L.Opening.clear(), L.Opening.bit_dropped(suite.dropped_bits)):
            params = L.Params.sized(suite, opening)
            n = params.witness_len()
            pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
            w = L.Witness.random(pp, WITNESS_SEED)
            prover, verifier = L.Prover(pp), L.Verifier(pp)
            c0, op0 = prover.commit(w)
            t = L.Transcript(DOMAIN)
            point = verifier.derive_evaluation_point(t, c0)
            ch = verifier.derive_folding_challenges(t, w.row_evaluate(point))
            prover.recycle(op0)
            chal = np.ascontiguousarray(ch.challenges)
            st = torch.cuda.ExternalStream(N.lbg_prover_stream(prover._h))

            def step():
                op = ctypes.c_void_p()
                check(N.lbg_commit(prover._h, w._h, None, None, None, ctypes.byref(op)))
                check(N.lbg_fold(prover._h, op, ptr(chal), len(chal), None))

            for _ in range(2):
                step()
            check(N.lbg_prover_sync(prover._h))
            ts = []
            for _ in range(steps):
                with torch.cuda.stream(st):
                    flush.zero_()
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(st)
                step()
                b.record(st)
                b.synchronize()
                ts.append(a.elapsed_time(b))
            ms = float(np.median(ts))
            out.append({"suite": suite.name[4:], "opening": opening.kind, "log2_n": params.witness_log_len,
                        "columns": params.columns(), "moduli": params.primes(),
                        "dropped_bits": params.dropped_bits(), "commit_fold_ms": ms, "elems_s": n / (ms / 1000)})
            del prover, verifier, w, pp
    # Params::basic(): the whole round, public API (host transcript) and device round
    params = L.Params.basic()
    pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
    w = L.Witness.random(pp, WITNESS_SEED)
    prover, verifier = L.Prover(pp), L.Verifier(pp)

    def api_round():
        c, op = prover.commit(w)
        t = L.Transcript(DOMAIN)
        point = verifier.derive_evaluation_point(t, c)
        w.mle_evaluate(point)
        row = w.row_evaluate(point)
        ch = verifier.derive_folding_challenges(t, row)
        prover.fold(op, ch)

    api_round()
    t0 = time.perf_counter()
    for _ in range(steps):
        api_round()
    api_ms = (time.perf_counter() - t0) * 1000 / steps
    b = Batch(pp, [params.column_log_len])
    b.witness_random([WITNESS_SEED])
    b.round(DOMAIN, copy=False)
    t0 = time.perf_counter()
    for _ in range(steps):
        b.round(DOMAIN, copy=False)
    dev_ms = (time.perf_counter() - t0) * 1000 / steps
    basic = {"suite": "basic", "log2_n": 18, "round_api_ms": api_ms, "round_device_ms": dev_ms,
             "round_api_elems_s": params.witness_len() / (api_ms / 1000),
             "round_device_elems_s": params.witness_len() / (dev_ms / 1000),
             "workload": "Params::basic(): commit, evaluation point, mle and row evaluation, folding challenges, "
                         "fold; host clock around the calls (results read back)"}
    return {"plain": out, "basic_round": basic}


def run_ntt_micro(steps, count=1 << 20, q=3889):
    """The 648-point forward transform and its inverse over all ring elements of a 2^22 witness
    (2^20 ring elements, q = 3889, coefficients uniform in [0, q) from a seeded generator), each
    timed alone with CUDA events (inputs 1.36 GB, far above L2). GB/s counts 1296 B read + 1296 B
    written per ring element and direction."""
    import torch

    from labinius_b200 import ntt

    g = torch.Generator(device="cuda").manual_seed(2026)
    a = torch.randint(0, q, (count, 648), dtype=torch.int16, device="cuda", generator=g)
    y = torch.empty_like(a)
    z = torch.empty_like(a)
    for _ in range(2):
        ntt.forward(q, a, y)
        ntt.inverse(q, y, z)
    torch.cuda.synchronize()
    if not torch.equal(z, a):
        raise RuntimeError("ntt648 round trip failed")
    res = {}
    for name, fn, src, dst in (("forward", ntt.forward, a, y), ("inverse", ntt.inverse, y, z)):
        ts = []
        for _ in range(steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record()
            fn(q, src, dst)
            e1.record()
            e1.synchronize()
            ts.append(e0.elapsed_time(e1))
        ms = float(np.median(ts))
        res[name] = {"ms": ms, "gbs": 2 * 1296 * count / (ms / 1000) / 1e9}
    return {"ring_elements": count, "q": q, **res,
            "bytes_per_ring_element": 2592, "workload": "all ring elements of a 2^22 witness, d = 648, q = 3889"}


def b128_claim(partials):
    """The trace's value at the switch's point from its partial evaluations, sum_k v_k x^k in B128
    (crates/pcs/src/switch.rs:116-122)."""
    acc = 0
    for k in range(127, -1, -1):
        acc <<= 1
        if acc >> 128:
            acc ^= (1 << 128) | 0x87
        acc ^= int(partials[k][0]) | (int(partials[k][1]) << 64)
    return np.array([acc & ((1 << 64) - 1), acc >> 64], np.uint64)


def run_switch(steps, sizes=(18, 20, 22)):
    """The cross-field switch prover (crates/pcs/src/switch.rs:65-74) through the API: a lifted B128
    trace of 2^l words (column length 2048), a point r and the trace's value there, switch::prove
    with the caller's transcript (moved to the device and back); host clock around the synchronous
    call, inputs resident."""
    import labinius_b200 as L
    from labinius_b200 import switch

    out = {}
    for wl in sizes:
        params = L.Params.new(wl, wl - 11, [L.Modulus.Q9721_FS_S])
        pp = L.PublicParameters.from_seed(params, MATRIX_SEED)
        rng = np.random.default_rng(wl)
        n = params.witness_len()
        trace = np.frombuffer(rng.bytes(16 * n), dtype=np.uint64).reshape(n, 2)
        r = np.frombuffer(rng.bytes(16 * wl), dtype=np.uint64).reshape(wl, 2)
        w = L.Witness.lifted(pp, trace)
        proof, _ = switch.prove(pp, w, r, np.zeros(2, np.uint64), L.Transcript(b"claim"))
        claim = b128_claim(proof.partials)
        switch.prove(pp, w, r, claim, L.Transcript(DOMAIN))
        ts = []
        for _ in range(steps):
            t0 = time.perf_counter()
            switch.prove(pp, w, r, claim, L.Transcript(DOMAIN))
            ts.append(time.perf_counter() - t0)
        ms = 1000 * float(np.median(ts))
        out[f"2^{wl}"] = {"ms": ms, "elems_s": n / (ms / 1000)}
        del w, pp
    out["workload"] = ("switch::prove of a lifted B128 trace at a random point, claim = the trace's value there; "
                       "median host-clock time of the synchronous API call")
    return out


def run_wire(L, prover, params, steps):
    """wire::encode of the prover's last folded witness (crates/pcs/src/wire/rans.rs:18-105): on the
    device from where Prover::fold left it, and through the host-memory entry point; the host clock
    around the synchronous calls; the size against the zeroth-order entropy."""
    from labinius_b200 import wire
    from labinius_b200._native import check, lib, ptr

    vv = np.zeros((params.len_ring(), 648), np.int16)
    check(lib().lbg_prover_folded(prover._h, ptr(vv)))
    data = wire.encode_folded(prover)
    dev, host = [], []
    for _ in range(steps):
        t0 = time.perf_counter()
        wire.encode_folded(prover)
        dev.append(time.perf_counter() - t0)
        t0 = time.perf_counter()
        wire.encode(vv, params.primes()[0])
        host.append(time.perf_counter() - t0)
    _, counts = np.unique(vv, return_counts=True)
    p = counts / counts.sum()
    entropy = float(-(counts * np.log2(p)).sum() / 8.0)
    return {"coefficients": int(vv.size), "bytes": len(data), "bits_per_coefficient": 8.0 * len(data) / vv.size,
            "entropy_bytes": entropy, "device_ms": 1000 * float(np.median(dev)),
            "host_input_ms": 1000 * float(np.median(host)),
            "workload": "the folded witness of the bench's step (len_ring x 648 int16), interleaved rANS, 64 lanes"}


def run_served(requests, plain_sample, load=0.7, slots=3, seed=2027, server_kw=None):
    """Served: commit+open requests with log2 n ~ U{18..22} (column length 2048, moduli [3889, 9721]),
    80% Witness::random and 20% B128 traces opened through the cross-field switch, each from its
    own seed, through the serving loop (continuous batching over three device arenas, transcripts on
    the device). First the saturated throughput (every request queued at once, a sample of the
    stream); then the Poisson stream of `requests` arrivals at `load` x that throughput, with
    p50/p99 latency from arrival to result. The comparison is the plain per-request path, one
    request after another, on a sample of the same requests, its witnesses (and the B128 claims)
    made before the clock starts: commit, evaluation point, row and mle evaluation, folding
    challenges, fold; for a B128 trace commit, the tagged commitment absorbed, switch::prove, row
    evaluation at its point, folding challenges, fold (crates/pcs/examples/two_fields.rs:176-194)."""
    import labinius_b200 as L
    from labinius_b200 import switch
    from labinius_b200.batch import Batch
    from labinius_b200.serve import Request, Server

    rng = np.random.default_rng(seed)
    logs = rng.integers(18, 23, requests)
    kinds = (rng.random(requests) < 0.2).astype(int)
    seeds = [rng.bytes(32) for _ in range(requests)]
    gaps = rng.exponential(1.0, requests)
    col_logs = [int(x) - 11 for x in logs]

    def params(c):
        return L.Params.new(11 + c, c, [L.Modulus.Q9721_FS_S])

    pp = L.PublicParameters.from_seed(params(7), MATRIX_SEED)
    # small requests (at most 2^20 F162) on a slot of their own, so that none waits behind large ones
    # three slots (one for small requests, two taking large ones first) of at most 2048 columns a batch
    # (one 2^22 request): a large request waits for at most one batch of large work per slot. Measured
    # at 0.7 load over 10,000 requests: two slots of 4096 columns p99 28 ms, three of 4096 25 ms, three
    # of 2048 23 ms, for 6% less saturated throughput than two of 4096.
    kw = dict(capacity_columns=2048, max_requests=64, slots=slots, host_threads=os.cpu_count() or 1,
              keep_results=False, small_log_len=9)
    kw.update(server_kw or {})
    srv = Server(pp, **kw)

    def run(idx, rate):
        reqs, t0 = [], time.perf_counter()
        due = 0.0
        for k, i in enumerate(idx):
            if rate:
                due += gaps[k] / rate
                d = t0 + due - time.perf_counter()
                if d > 0:
                    time.sleep(d)
            reqs.append(srv.submit(Request(col_logs[i], seeds[i], int(kinds[i]))))
        for r in reqs:
            r.wait()
        errs = [r.error for r in reqs if r.error]
        if errs:
            raise RuntimeError(errs[0])
        first = min(r.arrival for r in reqs)
        last = max(r.done for r in reqs)
        elems = sum(1 << int(logs[i]) for i in idx)
        lat = np.array([r.latency for r in reqs]) * 1000
        return elems / (last - first), len(idx) / (last - first), lat, np.array([int(logs[i]) for i in idx])

    run(range(min(64, requests)), None)  # warm-up: arenas, graphs of the host pool
    sat_n = min(requests, 2000)
    # the better of two saturated runs (a single one varied by a third between runs)
    sat_runs = [run(range(sat_n), None)[:2] for _ in range(2)]
    sat_elems, sat_reqs = max(sat_runs)
    rate = load * sat_reqs
    b0 = srv.batches
    st_elems, st_reqs, lat, lat_logs = run(range(requests), rate)
    batches = srv.batches - b0
    srv.close()
    if plain_sample == 0:
        return {"rate_req_s": rate, "batches": batches, "throughput_elems_s": st_elems,
                "saturated_elems_s": sat_elems, "p50_ms": float(np.percentile(lat, 50)),
                "p99_ms": float(np.percentile(lat, 99)),
                "by_log2_n": {str(lg): [float(np.percentile(lat[lat_logs == lg], 50)),
                                        float(np.percentile(lat[lat_logs == lg], 99))]
                              for lg in range(18, 23) if (lat_logs == lg).any()}}

    # the plain per-request path on a sample of the same requests
    pps = {}
    sample = list(range(min(plain_sample, requests)))
    wits, points, claims = [], {}, {}
    for i in sample:
        c = col_logs[i]
        if c not in pps:
            pps[c] = (L.PublicParameters.from_seed(params(c), MATRIX_SEED),)
            pps[c] += (L.Prover(pps[c][0]), L.Verifier(pps[c][0]))
        p = pps[c][0]
        if kinds[i]:
            # the trace a B128 front end would hold on the host (made by the device generator)
            g = Batch(p, [c])
            g.witness_random([seeds[i]], [1])
            wits.append(L.Witness.lifted(p, np.ascontiguousarray(g.elements(0)[:, :2])))
            del g
            points[i] = srv.switch_point(Request(col_logs[i], seeds[i], 1))
            proof, _ = switch.prove(p, wits[-1], points[i], np.zeros(2, np.uint64), L.Transcript(b"claim"))
            claims[i] = b128_claim(proof.partials)
        else:
            wits.append(L.Witness.random(p, seeds[i]))
    lat_plain, plain_logs = [], []
    t0 = time.perf_counter()
    for k, i in enumerate(sample):
        plain_logs.append(int(logs[i]))
        s0 = time.perf_counter()
        p, prover, verifier = pps[col_logs[i]]
        w = wits[k]
        c, op = prover.commit(w)
        t = L.Transcript(DOMAIN)
        if kinds[i]:
            t.absorb_bytes(c.to_bytes())
            _, point = switch.prove(p, w, points[i], claims[i], t)
        else:
            point = verifier.derive_evaluation_point(t, c)
            w.mle_evaluate(point)
        row = w.row_evaluate(point)
        ch = verifier.derive_folding_challenges(t, row)
        prover.fold(op, ch)
        lat_plain.append((time.perf_counter() - s0) * 1000)
    plain_s = time.perf_counter() - t0
    plain_elems = sum(1 << int(logs[i]) for i in sample) / plain_s
    lat_plain, plain_logs = np.array(lat_plain), np.array(plain_logs)
    by_size = {}
    for lg in range(18, 23):
        sel, psel = lat[lat_logs == lg], lat_plain[plain_logs == lg]
        by_size[str(lg)] = {"requests": int(len(sel)),
                            "p50_ms": float(np.percentile(sel, 50)) if len(sel) else None,
                            "p99_ms": float(np.percentile(sel, 99)) if len(sel) else None,
                            "plain_p50_ms": float(np.percentile(psel, 50)) if len(psel) else None,
                            "plain_p99_ms": float(np.percentile(psel, 99)) if len(psel) else None}
    return {"requests": requests, "rate_req_s": rate, "load": load, "batches": batches, "by_log2_n": by_size,
            "admission": "arenas within half the free HBM, at most %d columns a batch; requests of at most "
                         "2^20 F162 on a slot of their own (greatest stream priority), the other %d slots large "
                         "ones first" % (kw["capacity_columns"], slots - 1),
            "throughput_elems_s": st_elems, "throughput_req_s": st_reqs,
            "p50_ms": float(np.percentile(lat, 50)), "p99_ms": float(np.percentile(lat, 99)),
            "mean_ms": float(lat.mean()),
            "saturated_elems_s": sat_elems, "saturated_req_s": sat_reqs, "saturated_sample": sat_n,
            "saturated_runs_elems_s": [r[0] for r in sat_runs],
            "plain_elems_s": plain_elems, "plain_sample": len(sample),
            "plain_p50_ms": float(np.percentile(lat_plain, 50)), "plain_p99_ms": float(np.percentile(lat_plain, 99)),
            "speedup_saturated_vs_plain": sat_elems / plain_elems,
            "workload": "commit+open per request; log2 n ~ U{18..22}, column length 2048, moduli [3889, 9721]; "
                        "80% Witness::random (commit, evaluation point, mle and row evaluation, folding "
                        "challenges, fold), 20% B128 traces opened through the cross-field switch at a point "
                        "drawn from the request's seed (commit, tagged commitment absorbed, switch::prove of "
                        "the trace's value there, row evaluation, folding challenges, fold); Poisson "
                        "arrivals at load x saturated rate",
            "slots": slots, "slot_columns": kw["capacity_columns"], "host_threads": os.cpu_count() or 1}


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
    wseed = rank_witness_seed(rank)
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
    value = whole_job_value(world, n, ms_max)

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
    # transform: 54 level-2 radix-3 butterflies of one Shoup product, 9 ops, and 108 of three, 15
    # ops; 162 window lookups x 2; 162 reductions x 3; the module product: 648 multiply-adds)
    int_ops = n * (54 * 9 + 108 * 15 + 162 * 2 + 162 * 3 + 648)
    fold_ms = stats["fold"][1] / max(stats["fold"][0], 1)

    e2e = None
    if not args.no_e2e:
        host_w = torch.empty((n, 3), dtype=torch.int64, pin_memory=True)
        hw = host_w.numpy().view(np.uint64)
        hw[:] = w.elements()
        L_ = len(params.primes())
        mat = torch.empty((r, 4, L_, 162), dtype=torch.int16, pin_memory=True).numpy()
        vout = torch.empty((params.len_ring(), 648), dtype=torch.int16, pin_memory=True).numpy()

        # the same witness in ordinary pageable memory, as a Rust Vec<F162> or a numpy array is
        hw_pageable = np.array(hw, copy=True)
        mat_pageable = np.empty_like(mat)
        vout_pageable = np.empty_like(vout)

        def e2e_step(src=hw, m=mat, v=vout):
            # Witness::from_elements + Prover::commit (the upload pipelined against the commit by
            # column groups), then Prover::fold, results read back
            wh = ctypes.c_void_p()
            op = ctypes.c_void_p()
            check(N.lbg_commit_host(prover._h, ptr(src), n, ptr(m), None, None, ctypes.byref(wh), ctypes.byref(op)))
            check(N.lbg_fold(prover._h, op, ptr(chal), len(chal), ptr(v)))
            N.lbg_witness_free(wh)

        def timed_e2e(**kw):
            for _ in range(2):
                e2e_step(**kw)
            torch.cuda.synchronize()
            barrier(world)
            t0 = time.perf_counter()
            for _ in range(args.steps):
                e2e_step(**kw)
            torch.cuda.synchronize()
            return allreduce_max((time.perf_counter() - t0) * 1000.0 / args.steps, world, "cuda")

        e2e_ms = timed_e2e()
        e2e_pageable_ms = timed_e2e(src=hw_pageable, m=mat_pageable, v=vout_pageable)
        e2e = {"value": whole_job_value(world, n, e2e_ms), "unit": "elems/s", "ms_per_step": e2e_ms,
               "h2d_bytes_per_step": 24 * n + chal.nbytes, "d2h_bytes_per_step": mat.nbytes + vout.nbytes,
               "host_memory": "page-locked witness, commitment and folded-witness buffers",
               "pageable": {"value": whole_job_value(world, n, e2e_pageable_ms), "unit": "elems/s",
                            "ms_per_step": e2e_pageable_ms,
                            "host_memory": "ordinary pageable buffers (the witness staged through the prover's "
                                           "page-locked ring by host threads)"},
               "timing": "host wall clock around synchronous API calls, max over ranks"}

    # wire::encode of the folded witness (crates/bench/src/bin/labinius.rs:142, "encode folded
    # witness"): from where the fold left it, and from host memory
    wire_times = None
    if rank == 0 and not args.no_wire:
        wire_times = run_wire(L, prover, params, max(3, min(args.steps, 10)))

    # the verifier's side of the round (crates/bench/src/bin/labinius.rs:151-176), on the device:
    # fold_commitment, fold_row_evaluation, verify_evaluation, verify_opening (Clear)
    verifier_times = None
    if rank == 0:
        c1, op1 = prover.commit(w)
        t1 = L.Transcript(DOMAIN)
        pt1 = verifier.derive_evaluation_point(t1, c1)
        mle1, row1 = w.mle_evaluate(pt1), w.row_evaluate(pt1)
        ch1 = verifier.derive_folding_challenges(t1, row1)
        v1 = prover.fold(op1, ch1)

        def vstep():
            fc = verifier.fold_commitment(c1, ch1)
            fr = verifier.fold_row_evaluation(row1, ch1)
            verifier.verify_evaluation(pt1, mle1, row1)
            verifier.verify_opening(c1, ch1, pt1, L.OpeningMessage.clear(fc, v1, fr))

        vstep()
        vts = []
        for _ in range(10):
            tv0 = time.perf_counter()
            vstep()
            vts.append(time.perf_counter() - tv0)
        verifier_times = {"verify_ms": 1000 * float(np.median(vts)), "accepted": True,
                          "workload": "fold_commitment + fold_row_evaluation + verify_evaluation + verify_opening "
                                      "(Clear) at the bench's suite, host clock around each call, inputs from host "
                                      "memory, median of 10"}

    batched = None
    if not args.no_batched:
        batched = run_batched(args.batch_instances, max(3, min(args.steps, 5)))
    suites = None
    if not args.no_suites and rank == 0:
        suites = run_suites(max(3, min(args.steps, 5)))
    ntt_micro = None
    if not args.no_ntt:
        ntt_micro = run_ntt_micro(max(3, min(args.steps, 10)), count=args.ntt_count)
        for k in ("forward", "inverse"):
            ntt_micro[k]["frac_of_hbm"] = ntt_micro[k]["gbs"] / hbm
    switch_times = None
    if not args.no_switch and rank == 0:
        switch_times = run_switch(max(3, min(args.steps, 10)), tuple(int(x) for x in args.switch_sizes.split(",")))
    served = None
    if not args.no_served and rank == 0 and world == 1:
        served = run_served(args.served_requests, args.served_plain_sample)

    cpu = None
    parity = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # the device's commitment and folded witness of the step, through the public API with host
        # buffers (the e2e step's outputs, or one more step), against the oracle's whole step
        if e2e is None:
            c_dev, op_dev = prover.commit(w)
            gpu_C, gpu_v = c_dev.matrix, prover.fold(op_dev, ch).elements
        else:
            gpu_C, gpu_v = mat, vout
        cpu, oC, ov = cpu_baseline((params.witness_log_len, params.column_log_len, params.primes()),
                                   os.cpu_count() or 1, chal)
        parity = {"checked": True, "C": bool(np.array_equal(gpu_C, oC)), "v": bool(np.array_equal(gpu_v, ov)),
                  "columns": r, "ring_elements": params.len_ring(),
                  "what": "the step's commitment matrix (every column, every limb) and folded witness (every "
                          "ring element) from the device through the C ABI, against the oracle's whole step "
                          "with the same challenges"}

    props = torch.cuda.get_device_properties(local)
    int_peak = props.multi_processor_count * 128 * float(clk.get("sm_max_mhz") or 1965.0) * 1e6 / 1e12
    line = {
        "metric": METRIC, "value": value, "unit": "elems/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "u32 mod q / GF(2)", "data": "synthetic",
        "config": bench_config(args.config, params, world),
        "parity": parity,
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                     "peak_source": peak_src, "traffic": traffic, "kernel": "k_commit (one launch per limb)",
                     "per_launch_ms": per_launch_ms, "algorithmic_bytes_per_launch": algo_bytes,
                     "int_pipe": {"ops_per_launch": int_ops, "achieved_tops": int_ops / (per_launch_ms / 1000) / 1e12,
                                  "peak_tops": int_peak, "frac": int_ops / (per_launch_ms / 1000) / 1e12 / int_peak,
                                  "note": "integer-pipe bound; ops counted from the kernel's arithmetic; peak = "
                                          "SMs x 4 schedulers x 32 lanes x max SM clock (one 32-bit op per lane "
                                          "and cycle)"}},
        "kernels_ms": {k: {"launches": c, "avg_ms": (tt / c if c else None)} for k, (c, tt) in stats.items()},
        "t_commit_ms": stats["commit"][1] / args.steps + stats["commit_finish"][1] / args.steps,
        "t_fold_ms": (stats["fold"][1] + stats["challenge_slots"][1]) / args.steps,
        "t_fold_kernel_ms": fold_ms,
        "t_row_evaluate_ms": t_row * 1000, "t_mle_ms": t_mle * 1000,
        "gpu_launches": launches,
        "clocks": clk,
        "cpu_baseline": cpu,
        "e2e": e2e,
        "batched": batched,
        "served": served,
        "switch": switch_times,
        "wire": wire_times,
        "ntt_microbench": ntt_micro,
        "suites": suites,
        "verifier": verifier_times,
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

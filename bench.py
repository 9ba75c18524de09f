#!/usr/bin/env python
"""Benchmark of the Binius64 prove entry on B200.

Default workload (one "step" = one whole proof): Prover::prove of a synthetic constraint system
with 2^20 committed witness words, 2^20 - 2^16 AND constraints (padded to 2^20) and one MUL
constraint, log_inv_rate 1 -- the shape of the reference's sha512 64 KiB example (2^20 words,
2^20 ANDs, 1 intmul), whose constraint system cannot be built here (it comes from the Rust
frontend).  Operands are XORs of 1-3 shifted witness words over all eight shift variants, the
witness is seeded random and satisfies every constraint.  Proof parameters come from
Verifier::setup: 2^19 packed elements, 16 interleaved columns, fold arities [4, 4], 232 queries.

value: milliseconds per proof with the witness resident in HBM (CUDA events around each proof on
the proving stream; a 256 MiB buffer is written between proofs to flush L2).  e2e: the same proof
through the public API with the witness copied from pinned host memory inside the timed region;
the proof bytes (assembled on the host) are the result.  roofline: the dominant kernel of the
proof (the bivariate product sumcheck fold + round, shift phase 2 and BaseFold) timed live on
2^20-element operands.

--workload commit: the kernel-level FRI commit pipeline (RS encode of 16 interleaved columns of
codeword length 2^20, SHA-256 Merkle commit, 3 FRI folds with commits) with the NTT pass roofline.

--workload witness: witness generation on the device (the frontend's evaluation-form bytecode)
for the same 2^20-word circuit, over a batch of instances with different witness inputs; value =
ms per instance with the inputs resident, e2e with the inputs copied in and every generated
witness copied out.

--impl reference times the CPU restatement of the reference (oracle/, all host threads) on the
same workload; the Rust reference cannot be built in this image (no cargo).
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

SEED = 20241203
LOG_INV_RATE = 1

# prove workload
LOG_WORDS = 20
MERKLE_HASH = "sha256"  # or "vision4": the `-c vision4` setup, every commitment a Vision-4 tree

# commit workload
LOG_LEN = 20          # per-column codeword length 2^20
LOG_BATCH = 4         # 16 interleaved columns
FOLD_ARITY = 4
N_FOLDS = 3

PROVE_METRIC = "prove ms @2^20 words"
PUBLISHED_REFERENCE_MS = 128.58  # the reference README's sha512 64 KiB prove, hardware unstated
WITNESS_METRIC = "witness generation ms per instance @2^20 words"
WITNESS_BATCH = 32
COMMIT_METRIC = "FRI commit ms: RS encode + SHA-256 Merkle + 3 FRI folds with commits"


def n_and_for(log_words):
    return (1 << log_words) - (1 << (log_words - 4))


def prove_config(log_words):
    return {
        "workload": f"Prover::prove, synthetic AND/MUL constraint system with 2^{log_words} "
                    f"committed words, {n_and_for(log_words)} AND constraints (padded to "
                    f"2^{log_words}), 1 MUL, log_inv_rate {LOG_INV_RATE}",
        "log_words": log_words, "n_and": n_and_for(log_words), "n_mul": 1,
        "log_inv_rate": LOG_INV_RATE, "security_bits": 96,
        "stand_in_for": "sha512 example circuit, 64 KiB message (2^20 words, 2^20 ANDs, 1 MUL)",
        "l2": "256 MiB buffer written between timed proofs (L2 flush)",
        "merkle_hash": MERKLE_HASH,
        "seed": SEED,
    }


def commit_config():
    log_dim = LOG_LEN - LOG_INV_RATE
    return {
        "workload": f"kernel-level FRI commit, log_len={LOG_LEN} per column, R={LOG_INV_RATE}, "
                    f"{1 << LOG_BATCH} interleaved columns, {N_FOLDS} folds (arity {FOLD_ARITY})",
        "log_len": LOG_LEN, "log_inv_rate": LOG_INV_RATE, "batch_columns": 1 << LOG_BATCH,
        "message_elems": 1 << (log_dim + LOG_BATCH), "codeword_elems": 1 << (LOG_LEN + LOG_BATCH),
        "l2": "inputs larger than L2 (128 MiB message, 256 MiB codeword); no flush",
        "seed": SEED,
    }


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="prove",
                    choices=["prove", "commit", "batch", "serve", "witness"])
    ap.add_argument("--requests", type=int, default=256, help="batch / serve: proofs submitted")
    ap.add_argument("--workers", type=int, default=16, help="batch / serve: proving threads")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-batch", action="store_true",
                    help="prove workload: skip the batched-queue summary (profiling runs)")
    ap.add_argument("--tuning", default="",
                    help="launch shapes to set instead of autotuning, e.g. "
                         "'tail_log=10,ntt_tile_bits=10' (implies --no-autotune)")
    ap.add_argument("--no-autotune", action="store_true",
                    help="prove workload: time the default launch shapes")
    ap.add_argument("--no-matrix", action="store_true",
                    help="prove workload: skip the kernel-level commit matrix summary")
    ap.add_argument("--log-words", type=int, default=None,
                    help="prove workload: log2 committed words (default 20)")
    ap.add_argument("--merkle-hash", default="sha256", choices=["sha256", "vision4"],
                    help="prove workload: Merkle hash of the commitments (default sha256; "
                         "vision4 skips the batched summary)")
    ap.add_argument("--log-len", type=int, default=None,
                    help="commit workload: per-column codeword log length (default 20)")
    args = ap.parse_args()
    global LOG_WORDS, LOG_LEN, MERKLE_HASH
    MERKLE_HASH = args.merkle_hash
    if args.log_words is not None:
        assert 8 <= args.log_words <= 22
        LOG_WORDS = args.log_words
    if args.log_len is not None:
        assert 13 <= args.log_len <= 24
        LOG_LEN = args.log_len
    args.warmup = max(3, args.warmup)
    return args


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def max_over_ranks(value: float, pg, device: str) -> float:
    """The largest of every rank's value (replicas: the job ends when its slowest rank does);
    the value itself with one rank (pg None).  device: where the collective's tensor lives
    ("cuda:i" under NCCL, "cpu" under gloo)."""
    if pg is None:
        return value
    import torch
    pg.barrier()
    t = torch.tensor([value], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def whole_job_ms_per_unit(slowest_ms: float, units_per_rank: int, world: int) -> float:
    """Whole-job time per unit (proof, instance) for weak-scaled replicas: every rank processes
    units_per_rank units in parallel, so the job does units_per_rank * world units in the
    slowest rank's time."""
    return slowest_ms / (units_per_rank * world)


def fold_challenges(rng, n):
    return rng.integers(0, np.iinfo(np.uint64).max, size=(n, 2), dtype=np.uint64, endpoint=True)


# ----------------------------------------------------------------------------- clocks / peaks

def sample_clocks_start(device):
    """Starts nvidia-smi sampling every 50 ms and waits (up to 3 s) for its first sample, so
    that the region measured next is covered from its start."""
    try:
        f = tempfile.NamedTemporaryFile(prefix="clocks_", suffix=".csv", delete=False)
        p = subprocess.Popen(
            ["nvidia-smi", "-i", str(device),
             "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
             "--format=csv,noheader,nounits", "-lms", "50"],
            stdout=f, stderr=subprocess.DEVNULL)
        t0 = time.perf_counter()
        while time.perf_counter() - t0 < 3.0 and os.path.getsize(f.name) == 0:
            time.sleep(0.02)
        return p, f.name
    except (OSError, FileNotFoundError):
        return None, None


def sample_clocks_stop(handle):
    p, path = handle
    if p is None:
        return None
    p.terminate()
    try:
        p.wait(timeout=5)
    except subprocess.TimeoutExpired:
        p.kill()
    sm, mx, reasons = [], None, set()
    names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
    try:
        for line in open(path):
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
        os.unlink(path)
    except OSError:
        return None
    if not sm:
        return None
    return {"sm_mhz": statistics.median(sm), "sm_max_mhz": mx, "reasons": sorted(reasons),
            "samples": len(sm)}


def measured_peak_hbm():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def profiled_traffic(name):
    """dram bytes per launch from a committed ncu summary under profiles/, if present."""
    try:
        for line in open(os.path.join(ROOT, "profiles", name)):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1].strip())
    except (OSError, ValueError):
        pass
    return None


def pct(xs, q):
    xs = sorted(xs)
    k = min(len(xs) - 1, max(0, int(round(q / 100.0 * (len(xs) - 1)))))
    return xs[k]


# ----------------------------------------------------------------------------- prove workload

def make_circuit(log_words):
    from binius64_b200 import constraint_system as csm
    return csm.synthetic_circuit(log_words, n_and_for(log_words), 1, seed=SEED + log_words)


def cpu_prove_ms(circ, threads, reps=1):
    """Whole proofs on the oracle (C++ restatement of the reference); returns ms per proof."""
    import oracle as orc
    prep = circ.cs.prepared()
    orc.set_threads(threads)
    times = []
    with orc.merkle_hash(MERKLE_HASH):
        for _ in range(reps):
            t0 = time.perf_counter()
            orc.prove(circ.witness, 1, prep.and_csr, prep.mul_csr, LOG_INV_RATE)
            times.append(time.perf_counter() - t0)
    orc.set_threads(1)
    return 1000.0 * statistics.mean(times)


def vision4_kernels(torch, bg, device, stream):
    """Kernel-level Vision-4 figures (CUDA events around one call after a warm-up call): the
    permutation of 2^20 states, and the commit of the 2^20-word prove's codeword tree (2^16
    leaves of 16 elements)."""
    gen = torch.Generator(device=f"cuda:{device}").manual_seed(SEED)
    states = torch.randint(-2**63, 2**63 - 1, (4 << 20, 2), dtype=torch.int64,
                           device=f"cuda:{device}", generator=gen)
    elems = torch.randint(-2**63, 2**63 - 1, (1 << 20, 2), dtype=torch.int64,
                          device=f"cuda:{device}", generator=gen)
    mp = bg.BinaryMerkleTreeProver("vision4")
    out = {}
    for name, fn in (("permute_2^20_states_ms", lambda: bg.vision4_permute(states)),
                     ("commit_2^16_leaves_x16_ms", lambda: mp.commit(elems, 16))):
        fn()
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out[name] = e0.elapsed_time(e1)
    out["permutations_per_s"] = (1 << 20) / (out["permute_2^20_states_ms"] * 1e-3)
    return out


def bivariate_roofline(torch, bg, lib, device, stream, reps=20):
    """Live timing of binius_bivariate_fold_round_evals on 2^20-element operands (the first
    folded round of shift phase 2): algorithmic bytes = read a, b (2 x 16 MiB) + write the folded
    halves (2 x 8 MiB)."""
    log_len = 20
    n = 1 << log_len
    gen = torch.Generator(device=f"cuda:{device}").manual_seed(SEED)
    a0 = torch.randint(-2**63, 2**63 - 1, (n, 2), dtype=torch.int64, device=f"cuda:{device}",
                       generator=gen)
    b0 = torch.randint(-2**63, 2**63 - 1, (n, 2), dtype=torch.int64, device=f"cuda:{device}",
                       generator=gen)
    a, b = a0.clone(), b0.clone()
    out = torch.zeros((2, 2), dtype=torch.int64, device=f"cuda:{device}")
    r = (ctypes.c_uint8 * 16)(*range(1, 17))
    s = stream.cuda_stream
    for _ in range(3):
        a.copy_(a0)
        b.copy_(b0)
        lib.binius_bivariate_fold_round_evals(a.data_ptr(), b.data_ptr(), log_len, r,
                                                   out.data_ptr(), s)
    torch.cuda.synchronize()
    tot = 0.0
    for _ in range(reps):
        a.copy_(a0)
        b.copy_(b0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        lib.binius_bivariate_fold_round_evals(a.data_ptr(), b.data_ptr(), log_len, r,
                                                   out.data_ptr(), s)
        e1.record(stream)
        torch.cuda.synchronize()
        tot += e0.elapsed_time(e1)
    launch_ms = tot / reps
    bytes_per_launch = 2 * 16 * n + 2 * 16 * (n // 2)
    mults = n + n // 2  # n folds (both operands) + n/4 pairs x 2 products
    return launch_ms, bytes_per_launch, mults



# ----------------------------------------------------------------------------- batch / serve

BATCH_LOG_MIN, BATCH_LOG_MAX, BATCH_DISTINCT = 12, 20, 12


SERVE_EXTRA_LOG_WORDS = [21, 22]  # the served mix adds statements beyond the batched range


def mix_statement(torch, bg, device, lw, seed):
    """A synthetic statement of 2^lw words: AND chains over shifted operands plus
    2^(lw - 10) MUL constraints."""
    from binius64_b200 import constraint_system as csm
    n_mul = max(1, 1 << (lw - 10))
    sc = csm.synthetic_circuit(lw, n_and_for(lw) - 2 * n_mul, n_mul, seed=seed)
    prover = bg.Prover(bg.DeviceConstraintSystem(sc.cs.serialize(), device=device), LOG_INV_RATE)
    w = torch.from_numpy(sc.witness.view(np.int64)).to(f"cuda:{device}")
    return (lw, prover, w)


def batch_statements(torch, bg, device, n_distinct=BATCH_DISTINCT):
    """Distinct synthetic statements with log2(words) uniform in [12, 20] (log-uniform sizes)."""
    rng = np.random.default_rng(SEED + 7)
    sizes = sorted(int(x) for x in rng.integers(BATCH_LOG_MIN, BATCH_LOG_MAX + 1, size=n_distinct))
    return sizes, [mix_statement(torch, bg, device, lw, SEED + 100 + i)
                   for i, lw in enumerate(sizes)]


def autotune_statements(stmts):
    """Autotunes each distinct statement shape once (cached per shape by the library)."""
    for (lw, prover, w) in stmts:
        prover.autotune(w, reps=2)


def one_at_a_time(torch, stmts, order):
    """The requests proved back to back on one stream; returns (seconds, proofs by statement)."""
    proofs = {}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for i in order:
        pb = stmts[i][1].prove(stmts[i][2]).finalize()
        proofs.setdefault(i, pb)
    torch.cuda.synchronize()
    return time.perf_counter() - t0, proofs


def run_queue(bg, stmts, order, workers, arrivals=None):
    """Submits the requests (all at once, or at the given arrival offsets in seconds) to a
    ProveQueue; returns (seconds, latencies ms, prove ms, proofs in request order)."""
    q = bg.ProveQueue(n_workers=workers)
    tickets = []
    t0 = time.perf_counter()
    for k, i in enumerate(order):
        if arrivals is not None:
            delay = t0 + arrivals[k] - time.perf_counter()
            if delay > 0:
                time.sleep(delay)
        tickets.append(q.submit(stmts[i][1], stmts[i][2]))
    lat, prove, proofs = [], [], []
    for t in tickets:
        pb, tm = q.wait(t)
        lat.append(tm["latency_ms"])
        prove.append(tm["prove_ms"])
        proofs.append(pb)
    secs = time.perf_counter() - t0
    q.close()
    return secs, lat, prove, proofs


def batch_summary(torch, bg, device, n_requests, workers):
    sizes, stmts = batch_statements(torch, bg, device)
    rng = np.random.default_rng(SEED + 11)
    order = [int(x) for x in rng.integers(0, len(stmts), size=n_requests)]
    autotune_statements(stmts)
    for i in set(order):  # warm-up of every shape
        stmts[i][1].prove(stmts[i][2])
    t_seq, lone = one_at_a_time(torch, stmts, order)
    run_queue(bg, stmts, order[:64], workers)  # warm: the workers' arenas and the pool grow once
    t_q, lat, prove, proofs = run_queue(bg, stmts, order, workers)
    identical = all(proofs[k] == lone[i] for k, i in enumerate(order))
    return {
        "requests": n_requests, "workers": workers, "distinct_statements": len(stmts),
        "log_words": sizes, "proofs_per_s": n_requests / t_q,
        "one_at_a_time_proofs_per_s": n_requests / t_seq,
        "speedup_vs_one_at_a_time": t_seq / t_q,
        "latency_ms": {"p50": pct(lat, 50), "p99": pct(lat, 99)},
        "prove_ms_in_mix": {"p50": pct(prove, 50), "p99": pct(prove, 99)},
        "bit_identical_to_lone_proofs": identical,
    }, (sizes, stmts, order, t_seq, lone)


def serve_summary(torch, bg, device, batch_ctx, n_requests, workers):
    """A Poisson request stream (seeded arrivals) over the batched mix plus statements of 2^21
    and 2^22 words, at 70% of the queue's measured all-at-once capacity for this mix (the slower
    of two runs); latency
    percentiles, throughput, the one-at-a-time rate of the same requests and bit identity with
    the lone proofs."""
    sizes, stmts, _, _, _ = batch_ctx
    stmts = list(stmts)
    extra = [mix_statement(torch, bg, device, lw, SEED + 300 + k)
             for k, lw in enumerate(SERVE_EXTRA_LOG_WORDS)]
    autotune_statements(extra)
    stmts += extra
    sizes = [st[0] for st in stmts]
    rng = np.random.default_rng(SEED + 17)
    order = [int(x) for x in rng.integers(0, len(stmts), size=n_requests)]
    for i in set(order):
        stmts[i][1].prove(stmts[i][2])
    t_seq, lone = one_at_a_time(torch, stmts, order)
    run_queue(bg, stmts, order[:64], workers)  # warm: the workers' arenas and the pool grow once
    # capacity: the slower of two all-at-once runs (one run's estimate varies by ~10%, and an
    # optimistic one would put the Poisson stream above what the queue sustains)
    t_cap = max(run_queue(bg, stmts, order, workers)[0] for _ in range(2))
    rate = 0.7 * n_requests / t_cap
    arrivals = np.cumsum(np.random.default_rng(SEED + 13).exponential(1.0 / rate,
                                                                       size=n_requests)).tolist()
    t_q, lat, prove, proofs = run_queue(bg, stmts, order, workers, arrivals)
    identical = all(proofs[k] == lone[i] for k, i in enumerate(order))
    by_size = {}
    for k, i in enumerate(order):
        by_size.setdefault(sizes[i], []).append(lat[k])
    return {
        "requests": n_requests, "workers": workers, "log_words": sizes,
        "arrival_rate_per_s": rate, "capacity_proofs_per_s": n_requests / t_cap,
        "proofs_per_s": n_requests / t_q,
        "one_at_a_time_proofs_per_s": n_requests / t_seq,
        "capacity_vs_one_at_a_time": t_seq / t_cap,
        "latency_ms": {"p50": pct(lat, 50), "p99": pct(lat, 99), "max": max(lat)},
        "latency_ms_p99_by_log_words": {str(k): pct(v, 99) for k, v in sorted(by_size.items())},
        "prove_ms_in_mix": {"p50": pct(prove, 50), "p99": pct(prove, 99)},
        "bit_identical_to_lone_proofs": identical,
    }


def run_batch_workload(args, rank, world, local, serve=False):
    import torch
    import binius64_b200 as bg
    from binius64_b200._ffi import lib

    torch.cuda.set_device(local)
    if rank != 0:
        return
    clk = sample_clocks_start(local)
    launches0 = lib().binius_launch_count()
    summ, (sizes, stmts, order, t_seq, lone) = batch_summary(torch, bg, local, args.requests,
                                                             args.workers)
    line = {
        "metric": "batched proofs/s" if not serve else "served proofs/s (Poisson arrivals)",
        "unit": "proofs/s", "n_gpus": 1, "steps": args.requests, "warmup": len(set(order)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "GF(2^128) GHASH / u64 words",
        "data": "synthetic statements, log2(words) uniform in [12, 20], seeded",
        "config": {"workload": "independent proofs of a seeded mix of synthetic AND/MUL "
                               "constraint systems (2^12..2^20 words) through ProveQueue",
                   "requests": args.requests, "workers": args.workers, "log_words": sizes},
    }
    if not serve:
        line.update({"value": summ["proofs_per_s"], "ms_per_step": 1000.0 / summ["proofs_per_s"],
                     "batch": summ})
    else:
        sv = serve_summary(torch, bg, local, (sizes, stmts, order, t_seq, lone), args.requests,
                           args.workers)
        line["config"]["log_words"] = sv["log_words"]
        line["data"] = "synthetic statements, log2(words) in [12, 22], seeded"
        line.update({"value": sv["proofs_per_s"], "ms_per_step": 1000.0 / sv["proofs_per_s"],
                     "serve": sv, "batch": summ})
    line["gpu_launches"] = int(round((lib().binius_launch_count() - launches0) / args.requests))
    line["e2e"] = {"value": line["value"], "unit": "proofs/s", "h2d_bytes_per_step": 0,
                   "d2h_bytes_per_step": 0}
    line["clocks"] = sample_clocks_stop(clk)
    print(json.dumps(line), flush=True)


def run_prove(args, rank, world, local):
    import torch
    import binius64_b200 as bg
    from binius64_b200._ffi import lib

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    stream = torch.cuda.current_stream()
    circ = make_circuit(LOG_WORDS)
    dcs = bg.DeviceConstraintSystem(circ.cs.serialize(), device=local)
    prover = bg.Prover(dcs, LOG_INV_RATE, merkle_hash=MERKLE_HASH)
    w = torch.from_numpy(circ.witness.view(np.int64)).to(f"cuda:{local}")
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    proof = None
    for _ in range(args.warmup):
        proof = prover.prove(w).finalize()
    torch.cuda.synchronize()
    # the autotuner picks this statement shape's launch shapes (tail size, NTT layers per pass,
    # Merkle fusion; the proof bytes are unchanged) before anything is timed
    tuning = None
    if args.tuning:
        prover.set_tuning(**{k: int(v) for k, v in
                             (kv.split("=") for kv in args.tuning.split(",") if kv)})
        tuning = prover.tuning()
        assert prover.prove(w).finalize() == proof, "proof differs under the given launch shapes"
    elif not args.no_autotune:
        t_at = time.perf_counter()
        tuning = prover.autotune(w, reps=3)
        tuning["autotune_s"] = time.perf_counter() - t_at
        assert prover.prove(w).finalize() == proof, "autotuned proof differs"
    # set-up (context warm): ConstraintSystem parse + device upload + shift term table, prover
    # parameters and NTT twiddles; and the KeyCollection bytes (build_key_collection + serialize)
    cs_bytes = circ.cs.serialize()
    t_s0 = time.perf_counter()
    dcs2 = bg.DeviceConstraintSystem(cs_bytes, device=local)
    prover2 = bg.Prover(dcs2, LOG_INV_RATE, merkle_hash=MERKLE_HASH)
    torch.cuda.synchronize()
    t_s1 = time.perf_counter()
    bg.key_collection_from_cs_bytes(cs_bytes)
    t_s2 = time.perf_counter()
    setup = {"setup_ms": 1000.0 * (t_s1 - t_s0), "key_collection_ms": 1000.0 * (t_s2 - t_s1)}
    del prover2, dcs2

    # --- device-resident witness: CUDA events around each proof
    launches0 = lib().binius_launch_count()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clk = sample_clocks_start(local)
    per, phases = [], []
    t_wall0 = time.perf_counter()
    for _ in range(args.steps):
        flush.fill_(1)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        prover.prove(w)
        e1.record(stream)
        torch.cuda.synchronize()
        per.append(e0.elapsed_time(e1))
        phases.append(prover.phase_ms())
    wall = time.perf_counter() - t_wall0
    clocks = sample_clocks_stop(clk)
    launches = (lib().binius_launch_count() - launches0) / args.steps
    total_ms = max_over_ranks(sum(per), pg, f"cuda:{local}")
    ms = whole_job_ms_per_unit(total_ms, args.steps, world)  # whole-job ms per proof

    # --- end to end through the C ABI with host buffers (binius_prove): the witness words in
    # pinned host memory are copied in, the proof bytes come back into a host buffer; the same
    # warm-up count as the device-timed loop, then the same number of timed proofs
    host_w = torch.from_numpy(circ.witness.view(np.int64)).pin_memory()
    host_words = host_w.numpy().view(np.uint64)
    e2e = []
    proof_len = 0
    for k in range(args.warmup + args.steps):
        flush.fill_(1)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        pb = prover.prove_host(host_words, stream=stream)
        e1.record(stream)
        torch.cuda.synchronize()
        if k >= args.warmup:
            e2e.append(e0.elapsed_time(e1))
        proof_len = len(pb)
        assert pb == proof, "proof changed between runs"
    e2e_ms = statistics.mean(e2e)

    line = None
    if rank == 0:
        launch_ms, bpl, mults = bivariate_roofline(torch, bg, lib(), local, stream)
        achieved = bpl / (launch_ms * 1e-3) / 1e9
        peak, peak_kind = measured_peak_hbm()
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            threads = os.cpu_count() or 1
            cpu_ms = cpu_prove_ms(circ, threads, reps=2)
            cpu = {"value": cpu_ms, "unit": "ms", "cores": threads, "kind": "port",
                   "sample": f"2 whole proofs of the same 2^{LOG_WORDS}-word circuit on the "
                             "oracle (C++ restatement of the reference prover, PCLMULQDQ, "
                             "std::thread over all host cores); the Rust reference needs cargo"}
        kernels = vision4_kernels(torch, bg, local, stream) if MERKLE_HASH == "vision4" else None
        batched = served = matrix = None
        if world == 1 and not args.no_batch and MERKLE_HASH == "sha256":
            batched, ctx = batch_summary(torch, bg, local, 256, 16)
            served = serve_summary(torch, bg, local, ctx, 256, 16)
            del ctx
        if world == 1 and not args.no_matrix and MERKLE_HASH == "sha256":
            matrix = commit_matrix(torch, local, stream)
        ph = {k: statistics.median(p[k] for p in phases) for k in phases[0]}
        line = {
            "metric": PROVE_METRIC, "value": ms, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "GF(2^128) GHASH / u64 words", "data": "synthetic (seeded witness and "
            "constraint system of the reference's 2^20-word shape)",
            "config": prove_config(LOG_WORDS),
            "latency_ms": {"p50": pct(per, 50), "p99": pct(per, 99), "min": min(per),
                           "max": max(per), "wall_per_proof": 1000.0 * wall / args.steps},
            "phase_ms_host": ph,
            "setup": setup,
            "tuning": tuning,
            "batched": batched,
            "served": served,
            "commit_matrix": matrix,
            "vs_published_reference": {
                "reference_ms": PUBLISHED_REFERENCE_MS,
                "ratio_device": PUBLISHED_REFERENCE_MS / ms,
                "ratio_e2e": PUBLISHED_REFERENCE_MS / e2e_ms,
                "note": "the reference's own published prove time for the sha512 64 KiB "
                        "example (README.md, hardware unstated) over this line's 2^20-word "
                        "synthetic statement of the same shape: context, not a same-box ratio"},
            "vision4_kernels": kernels,
            "proof_bytes": proof_len,
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": int(host_w.numel() * 8),
                    "d2h_bytes_per_step": proof_len},
            "gpu_launches": int(round(launches)),
            "roofline": {"bound": "hbm", "kernel": "bivariate_fold_eval_kernel",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": profiled_traffic("bivariate_fold_eval_kernel_log20.md"),
                         "launch_ms": launch_ms, "algorithmic_bytes_per_launch": bpl,
                         "gf_mults_per_launch": mults,
                         "gf_mults_per_s": mults / (launch_ms * 1e-3),
                         "note": "GF(2^128) multiply-bound (integer pipes); HBM fraction "
                                 "reported against the measured copy bandwidth"},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- commit workload

C2_POINTS = [(L, R, b) for L in (20, 22, 24) for R in (1, 2) for b in (0, 4, 6)]


def commit_point(torch, device, stream, L, R, b, warm=3, reps=3, flush=None):
    """One point of the kernel-level FRI commit matrix: CUDA events around the encode, the
    Merkle commit and the 3 fold rounds of each timed run (a 256 MiB buffer is written between
    runs to flush L2).  Returns the point's figures."""
    from binius64_b200.commit_phase import CommitPhase
    ph = CommitPhase(L, R, b, seed=SEED + 1000 * L + 10 * R + b, device=device)
    for _ in range(warm):
        ph.run(stream)
    torch.cuda.synchronize()
    enc, mk, folds, step = [], [], [], []
    for _ in range(reps):
        if flush is not None:
            flush.fill_(1)
        marks = []
        ph.run(stream, marks)
        torch.cuda.synchronize()
        t = [marks[0].elapsed_time(m) for m in marks[1:]]
        enc.append(t[0])
        mk.append(t[1] - t[0])
        folds.append(t[-1] - t[1])
        step.append(t[-1])
    peak, _ = measured_peak_hbm()
    e, m, f, st = (statistics.mean(x) for x in (enc, mk, folds, step))
    out = {
        "log_len": L, "log_inv_rate": R, "columns": 1 << b,
        "codeword_bytes": 16 << (L + b),
        "step_ms": st, "encode_ms": e, "merkle_ms": m, "folds_ms": f,
        "encode_gbs": ph.encode_bytes() / (e * 1e-3) / 1e9,
        "merkle_gbs": ph.merkle_bytes() / (m * 1e-3) / 1e9,
        "encode_commit_gbs": ph.encode_commit_bytes() / ((e + m) * 1e-3) / 1e9,
        "step_gbs": ph.algorithmic_bytes() / (st * 1e-3) / 1e9,
        "ntt_gf_mults_per_s": ph.ntt_gf_mults() / (e * 1e-3),
        "sha256_compressions_per_s": ph.merkle_compressions() / (m * 1e-3),
    }
    out["encode_commit_frac"] = out["encode_commit_gbs"] / peak
    out["step_frac"] = out["step_gbs"] / peak
    ph.release()
    del ph
    torch.cuda.empty_cache()
    return out


def commit_matrix(torch, device, stream, points=C2_POINTS, warm=3, reps=3):
    """Every point of the C2 matrix, smallest first; peak HBM held: the largest point's buffers
    (25.3 GiB at log_len 24, R=1, 64 columns)."""
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{device}")
    res = [commit_point(torch, device, stream, L, R, b, warm, reps, flush)
           for (L, R, b) in sorted(points, key=lambda p: p[0] + p[2] - p[1])]
    peak, kind = measured_peak_hbm()
    return {"peak_gbs": peak, "peak_kind": kind, "warmup": warm, "reps": reps,
            "l2": "256 MiB buffer written between timed runs", "points": res}


def run_cpu_commit(threads):
    """The commit step on the CPU oracle (reference restatement); returns seconds."""
    import oracle as orc
    orc.set_threads(threads)
    log_dim = LOG_LEN - LOG_INV_RATE
    rng = np.random.default_rng(SEED)
    msg = orc.random_elems(rng, 1 << (log_dim + LOG_BATCH))
    tw = orc.domain_twiddles(LOG_LEN + LOG_BATCH)[: (1 << LOG_LEN) - 1]
    ch = [fold_challenges(rng, LOG_BATCH)] + [fold_challenges(rng, FOLD_ARITY)
                                               for _ in range(N_FOLDS - 1)]
    t0 = time.perf_counter()
    cw = orc.rs_encode_batch(tw, LOG_LEN, msg, log_dim, LOG_INV_RATE, LOG_BATCH)
    orc.merkle_commit(cw, LOG_LEN, LOG_BATCH)
    f = orc.fri_fold_interleaved(cw, LOG_LEN, LOG_BATCH, ch[0])
    orc.merkle_commit(f, LOG_LEN - FOLD_ARITY, FOLD_ARITY)
    cur = LOG_LEN
    for i in range(1, N_FOLDS):
        f = orc.fri_fold_codeword(tw, LOG_LEN, f, cur, ch[i])
        cur -= FOLD_ARITY
        orc.merkle_commit(f, cur - FOLD_ARITY, FOLD_ARITY)
    orc.set_threads(1)
    return time.perf_counter() - t0


def run_commit(args, rank, world, local):
    import torch
    from binius64_b200._ffi import lib
    from binius64_b200.commit_phase import CommitPhase

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    stream = torch.cuda.current_stream()
    pipe = CommitPhase(LOG_LEN, LOG_INV_RATE, LOG_BATCH, N_FOLDS, FOLD_ARITY, seed=SEED,
                       device=local)
    for _ in range(args.warmup):
        pipe.run(stream)
    torch.cuda.synchronize()
    launches0 = lib().binius_launch_count()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clk = sample_clocks_start(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        pipe.run(stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sample_clocks_stop(clk)
    launches = (lib().binius_launch_count() - launches0) / args.steps
    ms = whole_job_ms_per_unit(
        max_over_ranks(ev0.elapsed_time(ev1) / args.steps, pg, f"cuda:{local}"), 1, world)

    # dominant kernel: the NTT pass (ntt_pass_kernel launches over the codeword)
    reps = max(3, args.steps)
    for _ in range(2):
        pipe.ntt.forward_transform(pipe.codeword, LOG_INV_RATE, LOG_BATCH)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(reps):
        pipe.ntt.forward_transform(pipe.codeword, LOG_INV_RATE, LOG_BATCH)
    e1.record(stream)
    torch.cuda.synchronize()
    n_layers = LOG_LEN - LOG_INV_RATE
    n_passes = (n_layers + 7) // 8
    launch_ms = e0.elapsed_time(e1) / (reps * n_passes)
    bytes_per_launch = 32 * (1 << (LOG_LEN + LOG_BATCH))
    achieved = bytes_per_launch / (launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    mults_per_launch = (n_layers / n_passes) * (1 << (LOG_LEN + LOG_BATCH - 1))

    host_msg = torch.empty_like(pipe.message, device="cpu").pin_memory()
    host_msg.copy_(pipe.message.cpu())
    last = pipe.rounds[-1][3]
    host_out = torch.empty_like(last, device="cpu").pin_memory()
    trees = [pipe.nodes] + [r[4] for r in pipe.rounds]
    host_roots = torch.empty((len(trees), 32), dtype=torch.uint8).pin_memory()
    h2d = host_msg.numel() * 8
    d2h = host_out.numel() * 8 + host_roots.numel()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        pipe.message.copy_(host_msg, non_blocking=True)
        pipe.run(stream)
        host_out.copy_(last, non_blocking=True)
        for i, nd in enumerate(trees):
            host_roots[i].copy_(nd[-1], non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps
    pipe.release()
    del pipe
    torch.cuda.empty_cache()
    matrix = commit_matrix(torch, local, stream) if (world == 1 and args.log_len is None) else None

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cpu = {"value": run_cpu_commit(threads) * 1000.0, "unit": "ms", "cores": threads,
               "kind": "port", "sample": "one full step of the same workload on the oracle"}
    if rank == 0:
        line = {
            "metric": COMMIT_METRIC, "value": ms, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "GF(2^128) GHASH", "data": "synthetic (seeded uniform field elements)",
            "config": commit_config(),
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(round(launches)),
            "roofline": {"bound": "hbm", "kernel": "ntt_pass_kernel", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind,
                         "traffic": profiled_traffic("ntt_pass_kernel_log20_b4.md"),
                         "launch_ms": launch_ms, "algorithmic_bytes_per_launch": bytes_per_launch,
                         "gf_mults_per_launch": mults_per_launch,
                         "gf_mults_per_s": mults_per_launch / (launch_ms * 1e-3)},
            "matrix": matrix,
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


# ----------------------------------------------------------------------------- witness workload

def witness_setup(log_words):
    from binius64_b200 import eval_form as ef
    circ = make_circuit(log_words)
    code, n_values, n_insn = ef.synthetic_program(circ, with_count=True)
    return circ, code, n_values, n_insn, ef.synthetic_inputs(circ, n_values)


def witness_config(log_words, n_values, n_insn, batch):
    return {
        "workload": f"witness generation: the evaluation-form program recomputing the internal "
                    f"words of the 2^{log_words}-word synthetic circuit ({n_insn} instructions, "
                    f"{n_values} registers) for {batch} instances with different witness inputs",
        "log_words": log_words, "n_and": n_and_for(log_words), "n_mul": 1,
        "instructions": n_insn, "registers": n_values, "batch": batch,
        "l2": f"inputs larger than L2 ({n_values * batch * 8 >> 20} MiB of registers); no flush",
        "seed": SEED,
    }


DEEP_OPS = 1 << 17


def deep_chain_figures(torch, ef, dev, stream, args):
    """A deep program (chain_program: an add-rotate-xor chain of 2^17 instructions, levels a few
    instructions wide) for 1, 32 and 1024 instances: CUDA events around one evaluation after a
    warm-up one; the oracle's interpreter on one instance beside it."""
    code, n_values = ef.chain_program(DEEP_OPS, seed=SEED)
    prog = ef.EvalForm(code, n_values)
    out = {"instructions": prog.n_insn, "levels": prog.n_levels}
    for batch in (1, 32, 1024):
        regs = torch.zeros(n_values * batch, dtype=torch.int64, device=dev)
        regs[: 8 * batch] = 0x5A5A
        prog.evaluate(regs, batch)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        prog.evaluate(regs, batch)
        e1.record(stream)
        torch.cuda.synchronize()
        out[f"ms_batch_{batch}"] = e0.elapsed_time(e1)
    if not args.no_cpu_baseline:
        v0 = np.zeros(n_values, dtype=np.uint64)
        v0[:8] = 0x5A5A
        out["oracle_ms_one_instance"] = cpu_witness_ms(code, v0)
    return out


def cpu_witness_ms(code, v0, reps=1):
    import oracle as orc
    times = []
    for _ in range(reps):
        t0 = time.perf_counter()
        rc, _, _, _ = orc.eval_form_run(code, v0)
        times.append(time.perf_counter() - t0)
        assert rc == 0
    return 1000.0 * statistics.mean(times)


def run_witness(args, rank, world, local):
    import torch
    from binius64_b200 import eval_form as ef
    from binius64_b200._ffi import lib

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    stream = torch.cuda.current_stream()
    batch = WITNESS_BATCH
    circ, code, n_values, _, v0 = witness_setup(LOG_WORDS)
    prog = ef.EvalForm(code, n_values)
    lay = circ.cs.layout
    n_in, n_com = lay.committed_total_len - lay.n_internal, lay.committed_total_len
    rng = np.random.default_rng(SEED + 7)
    inputs = np.repeat(v0[None, :n_in], batch, axis=0)
    inputs[1:, lay.offset_witness:n_in] = rng.integers(
        0, 2**64, size=(batch - 1, n_in - lay.offset_witness), dtype=np.uint64, endpoint=False)
    dev = f"cuda:{local}"
    regs = torch.zeros(n_values * batch, dtype=torch.int64, device=dev)
    host_in = torch.from_numpy(inputs.view(np.int64)).reshape(-1).pin_memory()
    d_in = torch.empty_like(host_in, device=dev)
    d_out = torch.empty(batch * n_com, dtype=torch.int64, device=dev)
    host_out = torch.empty(batch * n_com, dtype=torch.int64).pin_memory()
    d_in.copy_(host_in)
    ef.transpose_words(d_in, batch, n_in, out=regs[: n_in * batch])
    for _ in range(args.warmup):
        fails, _ = prog.evaluate(regs, batch)
    torch.cuda.synchronize()
    assert int(fails.sum()) == 0
    launches0 = lib().binius_launch_count()
    if pg:
        pg.barrier()
    clk = sample_clocks_start(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        prog.evaluate(regs, batch)
    e1.record(stream)
    torch.cuda.synchronize()
    clocks = sample_clocks_stop(clk)
    launches = (lib().binius_launch_count() - launches0) / args.steps
    step_ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, pg, dev)
    ms = whole_job_ms_per_unit(step_ms, batch, world)  # whole-job ms per instance
    # end to end: inputs in from pinned host memory, every witness out
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        d_in.copy_(host_in, non_blocking=True)
        ef.transpose_words(d_in, batch, n_in, out=regs[: n_in * batch])
        prog.evaluate(regs, batch)
        ef.transpose_words(regs[: n_com * batch], n_com, batch, out=d_out)
        host_out.copy_(d_out, non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / (args.steps * batch)
    out = host_out.numpy().view(np.uint64).reshape(batch, n_com)
    assert np.array_equal(out[0], circ.witness), "instance 0 must regenerate the circuit witness"
    deep = deep_chain_figures(torch, ef, dev, stream, args) if rank == 0 else None
    line = None
    if rank == 0:
        peak, peak_kind = measured_peak_hbm()
        bytes_step = 8 * prog.n_accesses * batch
        achieved = bytes_step / (step_ms * 1e-3) / 1e9
        cpu = None
        if world == 1 and not args.no_cpu_baseline:
            cpu = {"value": cpu_witness_ms(code, v0), "unit": "ms", "cores": 1, "kind": "port",
                   "sample": "one instance on the oracle's interpreter (a restatement of "
                             "Interpreter::run, sequential like the reference's)"}
        line = {
            "metric": WITNESS_METRIC, "value": ms, "unit": "ms", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": step_ms,
            "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
            "dtype": "u64 words", "data": "synthetic (seeded witness inputs)",
            "config": witness_config(LOG_WORDS, n_values, prog.n_insn, batch),
            "levels": prog.n_levels,
            "deep_chain": deep,
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": int(host_in.numel() * 8),
                    "d2h_bytes_per_step": int(host_out.numel() * 8)},
            "gpu_launches": int(round(launches)),
            "roofline": {"bound": "hbm", "kernel": "eval_level_kernel (all levels of one step)",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "peak_kind": peak_kind,
                         "traffic": None, "algorithmic_bytes_per_step": bytes_step,
                         "note": "algorithmic bytes = 8 x register accesses x batch"},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
    if pg:
        pg.barrier()
        pg.destroy_process_group()
    if line:
        print(json.dumps(line), flush=True)


# ----------------------------------------------------------------------------- reference arm

def reference_arm(args, rank):
    """The reference's CPU path on the same workload: the oracle (C++ restatement, all host
    threads); rank 0 only."""
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    if args.workload == "prove":
        circ = make_circuit(LOG_WORDS)
        times = []
        for i in range(args.warmup + args.steps):
            t = cpu_prove_ms(circ, threads)
            if i >= args.warmup:
                times.append(t)
        metric, config = PROVE_METRIC, prove_config(LOG_WORDS)
        sample = f"each step one whole proof of the 2^{LOG_WORDS}-word circuit"
    elif args.workload == "witness":
        circ, code, n_values, n_insn, v0 = witness_setup(LOG_WORDS)
        times = []
        for i in range(args.warmup + args.steps):
            t = cpu_witness_ms(code, v0)
            if i >= args.warmup:
                times.append(t)
        metric = WITNESS_METRIC
        config = witness_config(LOG_WORDS, n_values, n_insn, WITNESS_BATCH)
        sample = "each step one instance on the oracle's interpreter (sequential, one thread)"
        threads = 1
    else:
        times = []
        for i in range(args.warmup + args.steps):
            t = 1000.0 * run_cpu_commit(threads)
            if i >= args.warmup:
                times.append(t)
        metric, config = COMMIT_METRIC, commit_config()
        sample = "each step the full commit workload"
    ms = statistics.mean(times)
    line = {
        "impl": "reference", "metric": metric, "value": ms, "unit": "ms", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "GF(2^128) GHASH / u64 words",
        "data": "synthetic", "config": config,
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": threads, "kind": "port",
                         "sample": sample + " on the oracle (C++ restatement of the reference; "
                                   "the Rust reference needs cargo, absent here)"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        reference_arm(args, rank)
        return
    if args.workload == "prove":
        run_prove(args, rank, world, local)
    elif args.workload in ("batch", "serve"):
        run_batch_workload(args, rank, world, local, serve=args.workload == "serve")
    elif args.workload == "witness":
        run_witness(args, rank, world, local)
    else:
        run_commit(args, rank, world, local)


if __name__ == "__main__":
    main()

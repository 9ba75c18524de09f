#!/usr/bin/env python
"""Benchmark of the kernel-level FRI commit pipeline on B200.

Workload (one "step"): the FRI commit path of the Binius64 prover at kernel level on seeded
uniform GF(2^128) input -- RS encode (additive NTT, R = 1) of 16 interleaved columns whose per-column
codeword length is 2^20, the SHA-256 Merkle commit of the 2^24-element codeword (leaves of 16
symbols), then 3 FRI folds, each followed by the Merkle commit of the folded codeword with coset
leaves of 16 symbols: fold_interleaved (4 challenges) -> 2^20, fold_codeword (4) -> 2^16,
fold_codeword (4) -> 2^12.  Mirrors fri::commit_interleaved + FRIFoldProver::execute_fold_round
(prover/prover/src/fri/{commit,fold}.rs).

value: device time per step (CUDA events, message resident in HBM).  e2e: the same step through the
public API with the message copied from pinned host memory and the roots plus the final folded
codeword copied back, inside the timed region.  Inputs (128 MiB message, 256 MiB codeword) exceed the
126 MB L2, so no explicit flush is needed between steps.

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

LOG_LEN = 20          # per-column codeword length 2^20
LOG_INV_RATE = 1
LOG_BATCH = 4         # 16 interleaved columns
FOLD_ARITY = 4
N_FOLDS = 3
SEED = 20241203

METRIC = "FRI commit ms: RS encode + SHA-256 Merkle + 3 FRI folds with commits"


def workload_config():
    log_dim = LOG_LEN - LOG_INV_RATE
    return {
        "workload": f"kernel-level FRI commit, log_len={LOG_LEN} per column, R={LOG_INV_RATE}, "
                    f"{1 << LOG_BATCH} interleaved columns, {N_FOLDS} folds (arity {FOLD_ARITY})",
        "log_len": LOG_LEN, "log_inv_rate": LOG_INV_RATE, "batch_columns": 1 << LOG_BATCH,
        "message_elems": 1 << (log_dim + LOG_BATCH), "codeword_elems": 1 << (LOG_LEN + LOG_BATCH),
        "field": "GF(2^128) GHASH", "hash": "SHA-256 leaves + Binius SHA-256 compression",
        "l2": "inputs larger than L2 (128 MiB message, 256 MiB codeword); no flush",
        "seed": SEED,
    }


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--log-len", type=int, default=None,
                    help="per-column codeword log length (default 20; smaller cases for profiling)")
    args = ap.parse_args()
    if args.log_len is not None:
        global LOG_LEN
        assert 13 <= args.log_len <= 24
        LOG_LEN = args.log_len
    return args


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return rank, world, local


def fold_challenges(rng, n):
    v = rng.integers(0, np.iinfo(np.uint64).max, size=(n, 2), dtype=np.uint64, endpoint=True)
    return v


def elem_ints(arr):
    return [int(a[0]) | (int(a[1]) << 64) for a in arr]


# ----------------------------------------------------------------------------- GPU pipeline

class GpuPipeline:
    """Preallocated buffers; one step = encode + commit + 3 x (fold + commit) via the C ABI."""

    def __init__(self, torch, device):
        import binius64_b200 as bg
        from binius64_b200._ffi import check, lib
        self.torch, self.bg, self.L, self.check = torch, bg, lib(), check
        self.device = device
        log_dim = LOG_LEN - LOG_INV_RATE
        self.log_dim = log_dim
        basis = bg.standard_domain_rs_basis(LOG_LEN + LOG_BATCH, LOG_BATCH, device=device)
        self.ntt = bg.AdditiveNTT(LOG_LEN, basis=basis, device=device)
        gen = torch.Generator(device=f"cuda:{device}").manual_seed(SEED)
        d = f"cuda:{device}"
        self.msg = torch.randint(-2**63, 2**63 - 1, (1 << (log_dim + LOG_BATCH), 2),
                                 dtype=torch.int64, device=d, generator=gen)
        self.codeword = torch.empty((1 << (LOG_LEN + LOG_BATCH), 2), dtype=torch.int64, device=d)
        self.nodes = [torch.empty(((2 << LOG_LEN) - 1, 32), dtype=torch.uint8, device=d)]
        self.folded = []
        cur = LOG_LEN
        for i in range(N_FOLDS):
            out_len = cur if i == 0 else cur - FOLD_ARITY
            self.folded.append(torch.empty((1 << out_len, 2), dtype=torch.int64, device=d))
            leaves = out_len - FOLD_ARITY
            self.nodes.append(torch.empty(((2 << leaves) - 1, 32), dtype=torch.uint8, device=d))
            cur = out_len
        rng = np.random.default_rng(SEED)
        self.ch = [fold_challenges(rng, LOG_BATCH)] + [fold_challenges(rng, FOLD_ARITY)
                                                        for _ in range(N_FOLDS - 1)]
        self.ch_ptrs = [c.ctypes.data_as(ctypes.c_void_p) for c in self.ch]

    def step(self, stream):
        L, chk = self.L, self.check
        s = stream.cuda_stream
        chk(L.binius_fri_commit_interleaved(self.ntt.handle, self.msg.data_ptr(), self.log_dim,
                                            LOG_INV_RATE, LOG_BATCH, self.codeword.data_ptr(),
                                            self.nodes[0].data_ptr(), None, s))
        chk(L.binius_fri_fold_interleaved(self.codeword.data_ptr(), LOG_LEN, LOG_BATCH,
                                          self.ch_ptrs[0], self.folded[0].data_ptr(), s))
        chk(L.binius_merkle_commit(self.folded[0].data_ptr(), LOG_LEN - FOLD_ARITY, FOLD_ARITY,
                                   self.nodes[1].data_ptr(), s))
        cur = LOG_LEN
        for i in range(1, N_FOLDS):
            chk(L.binius_fri_fold_codeword(self.ntt.handle, self.folded[i - 1].data_ptr(), cur,
                                           self.ch_ptrs[i], FOLD_ARITY, self.folded[i].data_ptr(),
                                           s))
            cur -= FOLD_ARITY
            chk(L.binius_merkle_commit(self.folded[i].data_ptr(), cur - FOLD_ARITY, FOLD_ARITY,
                                       self.nodes[i + 1].data_ptr(), s))

    def roots(self):
        return [bytes(n[-1].cpu().numpy().tobytes()) for n in self.nodes]


def sample_clocks_start(device):
    try:
        f = tempfile.NamedTemporaryFile(prefix="clocks_", suffix=".csv", delete=False)
        p = subprocess.Popen(
            ["nvidia-smi", "-i", str(device),
             "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
             "--format=csv,noheader,nounits", "-lms", "100"],
            stdout=f, stderr=subprocess.DEVNULL)
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


def profiled_traffic():
    """dram bytes per ntt_pass_kernel launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "ntt_pass_kernel_log20_b4.md")
    try:
        for line in open(path):
            if line.startswith("traffic_bytes_per_launch:"):
                return int(line.split(":")[1].strip())
    except (OSError, ValueError):
        pass
    return None


def run_cpu_pipeline(threads):
    """The same step on the CPU oracle (reference restatement); returns seconds."""
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
    return time.perf_counter() - t0


def reference_arm(args, rank):
    if rank != 0:
        return
    threads = os.cpu_count() or 1
    times = []
    for i in range(args.warmup + args.steps):
        t = run_cpu_pipeline(threads)
        if i >= args.warmup:
            times.append(t)
    ms = 1000.0 * statistics.mean(times)
    line = {
        "impl": "reference", "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False,
        "scaling": "weak", "vs_baseline": None, "dtype": "GF(2^128) (u128)", "data": "synthetic",
        "config": workload_config(),
        "cpu_baseline": {"value": ms, "unit": "ms", "cores": threads, "kind": "port",
                         "sample": "the full step, every step (oracle/ C++ restatement of the "
                                   "reference; the Rust reference needs cargo, absent here)"},
        "e2e": {"value": ms, "unit": "ms", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def main():
    args = parse_args()
    rank, world, local = dist_env()
    if args.impl == "reference":
        reference_arm(args, rank)
        return

    import torch
    import binius64_b200 as bg
    from binius64_b200._ffi import lib

    torch.cuda.set_device(local)
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist
    stream = torch.cuda.current_stream()
    pipe = GpuPipeline(torch, local)

    for _ in range(max(3, args.warmup)):
        pipe.step(stream)
    torch.cuda.synchronize()

    # --- device-timed region
    launches0 = lib().binius_launch_count()
    if pg:
        pg.barrier()
    torch.cuda.synchronize()
    clk = sample_clocks_start(local)
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    for _ in range(args.steps):
        pipe.step(stream)
    ev1.record(stream)
    torch.cuda.synchronize()
    clocks = sample_clocks_stop(clk)
    if pg:
        pg.barrier()
    launches = lib().binius_launch_count() - launches0
    ms = ev0.elapsed_time(ev1) / args.steps
    if pg:
        t = torch.tensor([ms], device=f"cuda:{local}")
        pg.all_reduce(t, op=pg.ReduceOp.MAX)
        ms = float(t.item())

    # --- dominant kernel: the NTT pass (3 launches of ntt_pass_kernel over the codeword)
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
    bytes_per_launch = 32 * (1 << (LOG_LEN + LOG_BATCH))  # read + write of every element
    achieved = bytes_per_launch / (launch_ms * 1e-3) / 1e9
    peak, peak_kind = measured_peak_hbm()
    mults_per_launch = (n_layers / n_passes) * (1 << (LOG_LEN + LOG_BATCH - 1))

    # --- end to end: pinned host message in, roots + final folded codeword out
    host_msg = torch.empty_like(pipe.msg, device="cpu").pin_memory()
    host_msg.copy_(pipe.msg.cpu())
    host_out = torch.empty_like(pipe.folded[-1], device="cpu").pin_memory()
    host_roots = torch.empty((len(pipe.nodes), 32), dtype=torch.uint8).pin_memory()
    h2d = host_msg.numel() * 8
    d2h = host_out.numel() * 8 + host_roots.numel()
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.steps):
        pipe.msg.copy_(host_msg, non_blocking=True)
        pipe.step(stream)
        host_out.copy_(pipe.folded[-1], non_blocking=True)
        for i, nd in enumerate(pipe.nodes):
            host_roots[i].copy_(nd[-1], non_blocking=True)
    e1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = e0.elapsed_time(e1) / args.steps

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        cpu_s = run_cpu_pipeline(threads)
        cpu = {"value": cpu_s * 1000.0, "unit": "ms", "cores": threads, "kind": "port",
               "sample": "one full step of the same workload on the oracle (C++ restatement of "
                         "the reference, PCLMULQDQ, std::thread over all host cores)"}

    if rank == 0:
        line = {
            "metric": METRIC, "value": ms, "unit": "ms", "n_gpus": world, "steps": args.steps,
            "warmup": max(3, args.warmup), "ms_per_step": ms, "higher_is_better": False,
            "scaling": "weak", "vs_baseline": None, "dtype": "GF(2^128) (u128)",
            "data": "synthetic (seeded uniform field elements)", "config": workload_config(),
            "e2e": {"value": e2e_ms, "unit": "ms", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": int(launches),
            "roofline": {"bound": "hbm", "kernel": "ntt_pass_kernel", "achieved": achieved,
                         "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "traffic": profiled_traffic(),
                         "launch_ms": launch_ms, "algorithmic_bytes_per_launch": bytes_per_launch,
                         "gf_mults_per_launch": mults_per_launch,
                         "gf_mults_per_s": mults_per_launch / (launch_ms * 1e-3)},
            "cpu_baseline": cpu,
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    if pg:
        pg.barrier()
        pg.destroy_process_group()


if __name__ == "__main__":
    main()

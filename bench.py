#!/usr/bin/env python
"""Determinant-pair microbenchmark on B200: one step = one structure H/S evaluation.

Workload (the reference's determinant-pair microbenchmark shape): n_active = 14 orbitals,
7 alpha + 7 beta electrons, all C(14,7) = 3432 covalent determinants, the 429 covalent Rumer
structures, 11,778,624 ordered determinant pairs per evaluation; seeded synthetic S, h and
(ij|kl) = sum_P B_ij^P B_kl^P with B of shape [42, 14, 14] (vbcore.workloads.active_space).

Arms:
  default            the vbcore CUDA path (one process per GPU; N > 1 runs independent replicas,
                     the path has no data-path collective: "scaling": "weak").
  --impl reference   the CPU oracle (a port of the reference CPU path) on the host cores, on a
                     bounded sample of the same workload per step; rank 0 only.

value  = ordered determinant pairs evaluated per second, whole job, inputs resident in HBM;
e2e    = the same through the host-pointer API (pinned host inputs copied in, H and S copied
         back every step);
roofline = the dominant kernel (by CUDA-event phase time) against the FP64 peak measured here
         with cuBLAS DGEMM, using the pair-flop model per processed unit.
"""

from __future__ import annotations

import argparse
import glob
import json
import math
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "xmvb-cpp_b200"))

N_ACTIVE = 14
N_ELECTRONS = 14
N_AUX = 42  # 3 n_active auxiliary functions
SEED = 20261203
KEYWORD = "COV"


def flops_spin_pair(k: int) -> float:
    """Pair-flop model v1, per spin pair: LU (2/3 k^3) + inverse (4/3 k^3) + 1e (2 k^2) + 2e (6 C(k,2)^2)."""
    return (2.0 / 3.0) * k ** 3 + (4.0 / 3.0) * k ** 3 + 2.0 * k ** 2 + 6.0 * math.comb(k, 2) ** 2


def flops_full_pair(ka: int, kb: int) -> float:
    """Pair-flop model v1, per determinant pair: opposite-spin 2 ka^2 kb^2 + 6."""
    return 2.0 * ka * ka * kb * kb + 6.0


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


def config_dict(n_det, n_str, world):
    k = N_ELECTRONS // 2
    return {
        "workload": f"determinant-pair microbenchmark: n_active={N_ACTIVE}, {k}a+{k}b electrons, {n_det} covalent "
                    f"determinants, {n_str} covalent Rumer structures, {n_det * n_det:,} ordered determinant pairs "
                    "per H/S evaluation",
        "n_active": N_ACTIVE, "n_alpha": k, "n_beta": k, "n_determinants": n_det, "n_structures": n_str,
        "n_aux": N_AUX, "seed": SEED, "structure_class": KEYWORD,
        "l2": "256 MiB device write between timed steps (plus a >2 GB per-step working set)",
        "parallelism": f"replicas{world}" if world > 1 else "single-gpu",
    }


class ClockSampler:
    """nvidia-smi clocks during the timed region."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index: int):
        self.gpu = gpu_index
        self.file = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.proc = None

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.QUERY}", "--format=csv,noheader,nounits",
                                          "-lms", "100"], stdout=self.file, stderr=subprocess.DEVNULL)
        except (OSError, FileNotFoundError):
            self.proc = None

    def stop(self):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()
        self.file.flush()
        self.file.seek(0)
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.file.read().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9 or not parts[0].isdigit() or int(parts[0]) != self.gpu:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(names, parts[5:9]):
                if flag.lower().startswith("active"):
                    reasons.add(name)
        self.file.close()
        os.unlink(self.file.name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_fp64_peak_tflops(torch, device) -> float:
    """Best-of-5 cuBLAS DGEMM 8192^3 on this GPU (the FP64 denominator)."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=device)
    b = torch.randn(n, n, dtype=torch.float64, device=device)
    for _ in range(2):
        torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        e1.synchronize()
        best = min(best, e0.elapsed_time(e1))
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def read_profile_traffic(kernel: str):
    """Per-launch DRAM bytes of `kernel` from the committed ncu summaries (profiles/*.md)."""
    pat = re.compile(r"^traffic_bytes_per_launch\s+(\S+)\s+(\d+)")
    for path in sorted(glob.glob(os.path.join(ROOT, "profiles", "*.md"))):
        for line in open(path):
            m = pat.match(line.strip())
            if m and m.group(1) == kernel:
                return int(m.group(2))
    return None


def _oracle():
    """The CPU oracle module (only the CPU-baseline leg and the reference arm use it)."""
    path = os.path.join(ROOT, "oracle")
    if path not in sys.path:
        sys.path.insert(0, path)
    import oracle

    oracle.build()
    return oracle


def cpu_baseline(ex_oracle, S, h, eri, n_pairs_ordered, seconds: float = 15.0):
    """Time the oracle on a bounded prefix of the unordered determinant pairs with all host
    threads; returns the ordered-pair rate and a description."""
    O = _oracle()
    threads = os.cpu_count() or 1
    n_det = ex_oracle.n_determinants
    total_unordered = n_det * (n_det + 1) // 2
    t0 = time.perf_counter()
    probe = min(total_unordered, 20000)
    O.structure_matrices(N_ACTIVE, ex_oracle, S, h, eri, threads=threads, pair_limit=probe)
    dt = max(time.perf_counter() - t0, 1e-6)
    sample = int(min(total_unordered, max(probe, probe * seconds / dt)))
    t0 = time.perf_counter()
    _, _, done = O.structure_matrices(N_ACTIVE, ex_oracle, S, h, eri, threads=threads, pair_limit=sample)
    dt = time.perf_counter() - t0
    ordered_equiv = done * (n_pairs_ordered / total_unordered)
    return {
        "value": ordered_equiv / dt, "unit": "ordered determinant pairs/s", "cores": threads, "kind": "port",
        "sample": f"{done} of {total_unordered} unordered determinant pairs (d <= e, column order) of the same "
                  f"workload, each with its spin-pair algebra and structure accumulation, {dt:.1f} s wall",
    }


def run_reference(args):
    rank, world, _ = dist_env()
    if rank != 0:
        return 0
    from vbcore import workloads

    O = _oracle()
    S, h, eri = workloads.active_space(N_ACTIVE, N_AUX, SEED)
    ex = O.expand(O.generate_structures(KEYWORD, N_ACTIVE, N_ELECTRONS), N_ELECTRONS)
    n_det = ex.n_determinants
    ordered = n_det * n_det
    total_unordered = n_det * (n_det + 1) // 2
    threads = os.cpu_count() or 1
    probe = min(total_unordered, 20000)
    t0 = time.perf_counter()
    O.structure_matrices(N_ACTIVE, ex, S, h, eri, threads=threads, pair_limit=probe)
    dt = max(time.perf_counter() - t0, 1e-6)
    budget = 90.0 / max(1, args.steps + args.warmup)
    sample = int(min(total_unordered, max(probe, probe * budget / dt)))
    for _ in range(args.warmup):
        O.structure_matrices(N_ACTIVE, ex, S, h, eri, threads=threads, pair_limit=sample)
    times = []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, _, done = O.structure_matrices(N_ACTIVE, ex, S, h, eri, threads=threads, pair_limit=sample)
        times.append(time.perf_counter() - t0)
    total = sum(times)
    rate = args.steps * done * (ordered / total_unordered) / total
    line = {
        "metric": "determinant-pair elements/s (structure H/S evaluation)", "value": rate,
        "unit": "ordered determinant pairs/s", "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
        "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
        "config": config_dict(n_det, ex.n_structures, 1),
        "cpu_baseline": {"value": rate, "unit": "ordered determinant pairs/s", "cores": threads, "kind": "port",
                         "sample": f"{done} of {total_unordered} unordered determinant pairs per step"},
        "e2e": {"value": rate, "unit": "ordered determinant pairs/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def run_vbcore(args):
    import numpy as np
    import torch
    import vbcore
    from vbcore import workloads

    rank, world, local = dist_env()
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    torch.cuda.set_device(local)
    device = torch.device("cuda", local)

    # --profile: a reduced HBM budget (smaller determinant-pair bands) and no side measurements,
    # so that one kernel of the full-size evaluation can be captured under a profiler
    ctx = vbcore.Context(local, (4 << 30) if args.profile else 0)
    rows = vbcore.generate_structures(KEYWORD, N_ACTIVE, N_ELECTRONS)
    ex = vbcore.expand_structures(rows, N_ELECTRONS)
    plan = vbcore.HsPlan(ctx, ex, N_ACTIVE)
    n_det, n_str = ex.n_determinants, ex.n_structures
    ordered = n_det * n_det
    S, h, eri = workloads.active_space(N_ACTIVE, N_AUX, SEED)
    stream = torch.cuda.Stream(device)
    torch.cuda.set_stream(stream)
    ctx.set_stream(stream.cuda_stream)

    dS = torch.tensor(np.ascontiguousarray(S.T), device=device)
    dh = torch.tensor(np.ascontiguousarray(h.T), device=device)
    de = torch.tensor(eri, device=device)
    dH = torch.empty((n_str, n_str), dtype=torch.float64, device=device)
    dSo = torch.empty((n_str, n_str), dtype=torch.float64, device=device)
    flush = torch.empty(256 * 1024 * 1024 // 8, dtype=torch.float64, device=device)

    peak = None if args.profile else measured_fp64_peak_tflops(torch, device)
    plan.enable_phase_timing(True)

    def step():
        plan.execute_device(dS.data_ptr(), dh.data_ptr(), de.data_ptr(), dH.data_ptr(), dSo.data_ptr())

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()

    sampler = ClockSampler(local)
    sampler.start()
    time.sleep(0.3)
    step_ms, phases = [], []
    for _ in range(args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        step()
        e1.record(stream)
        e1.synchronize()
        step_ms.append(e0.elapsed_time(e1))
        phases.append(plan.phase_times())
    torch.cuda.synchronize()
    clocks = sampler.stop()
    total_ms = sum(step_ms)
    if world > 1:
        t = torch.tensor([total_ms], device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        total_ms = float(t.item())
        torch.distributed.barrier()
    stats = plan.stats()
    value = ordered * args.steps * world / (total_ms * 1e-3)

    # end to end through the host-pointer API with pinned buffers
    pS = torch.tensor(np.ascontiguousarray(S.T)).pin_memory()
    ph = torch.tensor(np.ascontiguousarray(h.T)).pin_memory()
    pe = torch.tensor(eri).pin_memory()
    pH = torch.empty((n_str, n_str), dtype=torch.float64).pin_memory()
    pSo = torch.empty((n_str, n_str), dtype=torch.float64).pin_memory()
    for _ in range(0 if args.profile else max(1, args.warmup // 2)):
        plan.execute_host_pointers(pS.data_ptr(), ph.data_ptr(), pe.data_ptr(), pH.data_ptr(), pSo.data_ptr())
    e2e_ms = 0.0
    for _ in range(0 if args.profile else args.steps):
        flush.fill_(1.0)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        plan.execute_host_pointers(pS.data_ptr(), ph.data_ptr(), pe.data_ptr(), pH.data_ptr(), pSo.data_ptr())
        e1.record(stream)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    if world > 1:
        t = torch.tensor([e2e_ms], device=device)
        torch.distributed.all_reduce(t, op=torch.distributed.ReduceOp.MAX)
        e2e_ms = float(t.item())
    e2e_value = ordered * args.steps * world / (e2e_ms * 1e-3) if e2e_ms > 0 else None
    h2d = (2 * N_ACTIVE * N_ACTIVE + len(eri)) * 8
    d2h = 2 * n_str * n_str * 8

    # roofline of the dominant kernel (pair-flop model per processed unit)
    mean_phase = {k: statistics.mean(p[k] for p in phases) for k in vbcore.PHASES}
    k = N_ELECTRONS // 2
    n_strings = len(ex.alpha_strings)
    spin_units = n_strings * (n_strings + 1) // 2
    det_units = stats["determinant_pairs"]  # orbit representatives under the alpha/beta exchange
    kernels = {
        "spin_pairs": ("spin_pairs_fast", spin_units * flops_spin_pair(k), spin_units),
        "determinant_pairs": ("full_pairs_kernel", det_units * flops_full_pair(k, k), det_units),
    }
    dominant = max(kernels, key=lambda name: mean_phase[name])
    kname, flops, units = kernels[dominant]
    achieved = flops / (mean_phase[dominant] * 1e-3) / 1e12
    traffic = read_profile_traffic(kname)
    per_kernel = {name: {"ms": mean_phase[name], "tflops": f / (mean_phase[name] * 1e-3) / 1e12,
                         "frac": f / (mean_phase[name] * 1e-3) / 1e12 / peak if peak else None, "units": u}
                  for name, (_, f, u) in kernels.items()}
    # whole evaluation under the same pair-flop model (ordered spin pairs and determinant pairs)
    model_flops = ordered * (flops_spin_pair(k) + flops_full_pair(k, k))
    evaluation = {"flops_model": model_flops, "ms": total_ms / args.steps,
                  "tflops": model_flops / (total_ms / args.steps * 1e-3) / 1e12}
    evaluation["frac"] = evaluation["tflops"] / peak if peak else None

    if rank == 0:
        base = None
        if world == 1 and not args.profile:
            O = _oracle()
            ex_o = O.expand(O.generate_structures(KEYWORD, N_ACTIVE, N_ELECTRONS), N_ELECTRONS)
            base = cpu_baseline(ex_o, S, h, eri, ordered)
        line = {
            "metric": "determinant-pair elements/s (structure H/S evaluation)", "value": value,
            "unit": "ordered determinant pairs/s", "n_gpus": world, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": total_ms / args.steps, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded)", "config": config_dict(n_det, n_str, world),
            "roofline": {"bound": "fp64", "kernel": kname, "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                         "frac": achieved / peak if peak else None, "traffic": traffic,
                         "peak_source": "cuBLAS DGEMM 8192^3 measured in this run (of measured)",
                         "flops_per_launch": flops, "units_per_launch": units},
            "phases_ms": mean_phase, "kernels": per_kernel, "evaluation": evaluation,
            "cpu_baseline": base,
            "e2e": {"value": e2e_value, "unit": "ordered determinant pairs/s", "h2d_bytes_per_step": h2d,
                    "d2h_bytes_per_step": d2h},
            "gpu_launches": stats["kernel_launches"] * args.steps,
            "careful_spin_pairs": stats["careful_spin_pairs"],
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    plan.close()
    ctx.close()
    if world > 1:
        torch.distributed.destroy_process_group()
    return 0


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=30)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="vbcore", choices=["vbcore", "reference"])
    ap.add_argument("--profile", action="store_true",
                    help="for profiler captures: 4 GiB HBM budget, no DGEMM peak, CPU baseline or end-to-end leg")
    ap.add_argument("--n-active", type=int, default=14,
                    help="active orbitals (even; 14 is the benchmark workload, smaller cases are for profiling)")
    args = ap.parse_args()
    global N_ACTIVE, N_ELECTRONS, N_AUX
    if args.n_active != N_ACTIVE:
        if args.n_active % 2 or not 2 <= args.n_active <= 16:
            ap.error("--n-active must be even, 2..16")
        N_ACTIVE = N_ELECTRONS = args.n_active
        N_AUX = 3 * args.n_active
    if args.warmup < 3:
        args.warmup = 3
    if args.impl == "reference":
        return run_reference(args)
    return run_vbcore(args)


if __name__ == "__main__":
    sys.exit(main())

#!/usr/bin/env python
"""Benchmark of the distance-distribution hot path on B200.

Workload (default, `--workload an_k24`): the exact AN-code histogram for
A=58659 (16-bit odd constant), k=24 data bits: 40-bit codewords, all
2^24*(2^24-1)/2 = 140,737,479,966,720 unordered pairs, 41 uint64 bins.
One step = one full histogram through the C-ABI (dd_histogram).

Also measured (extra keys): the k=16 256-candidate super-A sweep as ONE
batched, graph-captured launch vs 256 one-launch-per-instance calls of the
persistent kernels and vs 256 plain one-launch-per-instance calls; the query
server on the seeded serving mix; the candidate pre-filter.  Outside the timed
region the headline histogram is computed once more on the other kernel and
must be identical (`parity`).

Reported per the harness contract: one JSON line on rank 0.
  value   pairs/s from the kernel's own CUDA events (codewords are generated
          on the device: the inputs are scalars already resident)
  e2e     pairs/s measured around the whole dd_histogram call on the stream
          (job-table H2D, bin reset, kernel, bins D2H)
  roofline  POPC-pipe fraction: pairs/s x popc-per-pair / measured POPC rate
  cpu_baseline  the reference's own CPU path (-c) on a bounded sample

`--impl reference` times the reference's own CPU implementation (its `codrel -c`
built from its sources) on the same workload metric, on a bounded sample.
Multi-GPU: replicas (each rank computes its own full instance; no collective).
"""
from __future__ import annotations

import argparse
import json
import os
import re
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path.insert(0, str(ROOT))

METRIC = "exact pairs/s (AN k=24 exhaustive histogram)"
NCU_DRAM_BYTES_PER_LAUNCH = 108288  # popc path: DRAM bytes of one launch, ncu capture at k=20
# tcgen05 path, by epilogue: DRAM bytes of one launch and sm__pipe_tensor_cycles_active
# of an ncu capture at k=20 (cold caches: the bytes are the job table, the bins and the
# kernel's own code; codewords are generated on chip)
NCU_DRAM_BYTES_PER_LAUNCH_MMA = {"paired": 136448, "single": 81408}
NCU_TENSOR_PIPE_PCT_MMA = {"paired": 12.1, "single": 16.9}
# instruction issue, the bound of the tcgen05 path's epilogue: warp instructions per
# pair (sm__inst_executed.sum / pairs of one k=20 launch; the single-epilogue capture
# recorded no count) and smsp__issue_active of the same captures
NCU_WARP_INST_PER_PAIR_MMA = {"paired": 5386.0 / 65536.0, "single": None}
NCU_ISSUE_ACTIVE_PCT_MMA = {"paired": 64.1, "single": 65.2}
ISSUE_PER_CLOCK_PER_SM = 4  # one warp instruction per clock from each of an SM's four schedulers
INT8_DENSE_TOPS_NOMINAL = 4500.0  # B200 dense int8 tensor rate (nominal; the measured peaks cover bf16 only)
MMA_K_PAD = 64  # int8 K of every tcgen05 tile (operand bit planes padded to 64)
UNIT = "pairs/s"


def issue_roofline(pairs_per_s: float, epilogue: str, sm_mhz, num_sms: int) -> dict:
    """Instruction issue of the tcgen05 path (the bound of its epilogue): warp
    instructions per pair from the ncu capture against 4 warp instructions per
    clock per SM at the sampled SM clock.  Fields are None where a figure is missing."""
    ipp = NCU_WARP_INST_PER_PAIR_MMA[epilogue]
    peak = ISSUE_PER_CLOCK_PER_SM * num_sms * (sm_mhz or 0) * 1e6
    return {"warp_inst_per_pair": ipp,
            "achieved_ginst_s": pairs_per_s * ipp / 1e9 if ipp else None,
            "peak_ginst_s": peak / 1e9 if peak else None,
            "frac": pairs_per_s * ipp / peak if ipp and peak else None,
            "ncu_issue_active_pct": NCU_ISSUE_ACTIVE_PCT_MMA[epilogue],
            "source": "warp instructions per pair from sm__inst_executed.sum of one k=20 ncu capture; peak = "
                      "4 warp instructions per clock per SM at the median SM clock sampled in the timed region"}


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=2)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="b200", choices=["b200", "reference"])
    p.add_argument("--workload", default="an_k24", choices=["an_k24", "an_k20", "an_k22"])
    p.add_argument("--kernel", default="auto", choices=["auto", "popc", "mma"])
    p.add_argument("--epilogue", default="auto", choices=["auto", "paired", "single"],
                   help="tcgen05 epilogue (auto: the autotuner's choice); pin it where a profiler's overhead "
                        "could change the autotuner's choice")
    p.add_argument("--launch-log", default="", help="write every launch's CUDA-event time (JSON) to this file")
    p.add_argument("--no-extras", action="store_true")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--no-parity", action="store_true", help="skip the cross-kernel check of the headline histogram")
    p.add_argument("--clocks-dir", default=os.environ.get("DD_CLOCKS_DIR", ""),
                   help="folder for the nvidia-smi clock samples of the timed region (default: temp dir)")
    return p.parse_args()


WORKLOADS = {"an_k24": (58659, 24), "an_k22": (58659, 22), "an_k20": (58659, 20)}


def pairs_of(n: int) -> int:
    N = 1 << n
    return N * (N - 1) // 2


# ------------------------------------------------------------------------------------
# clocks
# ------------------------------------------------------------------------------------
class ClockSampler:
    def __init__(self, index: int, path: Path):
        self.path = path
        self.proc = None
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.f = open(path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        self.f.close()
        sm, mx, reasons = [], None, set()
        for line in self.path.read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx = float(parts[2])
            except ValueError:
                continue
            names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
            for nm, v in zip(names, parts[5:9]):
                if v.lower().startswith("active"):
                    reasons.add(nm)
        busy = [s for s in sm if mx and s > 0.5 * mx] or sm
        return {"sm_mhz": statistics.median(busy) if busy else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


# ------------------------------------------------------------------------------------
# CPU baseline: the reference's own CPU path
# ------------------------------------------------------------------------------------
def cpu_baseline(A: int, budget_s: float = 20.0) -> dict:
    import oracle
    if oracle.ref_available():
        def run(n):
            out = oracle.ref_run(["-a", str(A), "-n", str(n), "-c"], timeout=600)
            return oracle.ref_total_runtime(out)
        kind = "reference"
    else:
        def run(n):
            t = time.perf_counter()
            oracle.an_exhaustive_raw(A, n, n + oracle.h_ceil(A) + 1)
            return time.perf_counter() - t
        kind = "port"
    n = 16
    t = run(n)
    # grow the sample (x4 pairs per +1 bit) while it stays inside the budget
    while t * 4 < 1.5 * budget_s and n < 24:
        n += 1
        t = run(n)
    return {"value": pairs_of(n) / t, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
            "sample": f"A={A}, k={n} exhaustive ({pairs_of(n)} pairs), `codrel -a {A} -n {n} -c`, "
                      f"OpenMP over all host cores, {t:.2f} s"}


def reference_arm(args) -> None:
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    import oracle
    A, k = WORKLOADS[args.workload]
    if not oracle.ref_available():
        kind = "port"
    else:
        kind = "reference"
    # bounded sample per step: the largest k whose run stays under ~6 s
    base = cpu_baseline(A, budget_s=6.0)
    n = int(re.search(r"k=(\d+)", base["sample"]).group(1))
    times = []
    for i in range(args.warmup + args.steps):
        if kind == "reference":
            out = oracle.ref_run(["-a", str(A), "-n", str(n), "-c"], timeout=600)
            t = oracle.ref_total_runtime(out)
        else:
            t0 = time.perf_counter()
            oracle.an_exhaustive_raw(A, n, n + oracle.h_ceil(A) + 1)
            t = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(t)
    tot = sum(times)
    v = pairs_of(n) * len(times) / tot
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": tot / len(times) * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "u64",
            "data": "synthetic", "config": {"workload": f"an_exhaustive_A{A}_k{k}", "A": A, "k": k,
                                              "sample_k": n, "cold_l2": "n/a (no memory traffic)"},
            "cpu_baseline": {"value": v, "unit": UNIT, "cores": os.cpu_count(), "kind": kind,
                             "sample": f"A={A}, k={n} exhaustive per step"},
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------
# replicas: one full instance per rank, no collective on the data path
# ------------------------------------------------------------------------------------
def max_over_ranks(values: list[float], world: int, device: str) -> list[float]:
    """Each value's maximum over all ranks (the slowest replica's times)."""
    if world == 1:
        return list(values)
    import torch
    import torch.distributed as dist
    t = torch.tensor(values, dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return t.tolist()


def replica_throughput(units_per_rank: int, world: int, slowest_ms: float) -> float:
    """Whole-job throughput: every rank processed units_per_rank units, the job
    ends with the slowest rank."""
    return units_per_rank * world / (slowest_ms * 1e-3)


def counts_digest(counts: list[int]) -> str:
    import hashlib
    return hashlib.sha256(",".join(str(c) for c in counts).encode()).hexdigest()


def cross_kernel_check(ctx, dd, A: int, k: int, timed) -> dict:
    """Recomputes the timed histogram on the other kernel (popc <-> tcgen05)
    and requires the identical raw bins and counts: two independent
    implementations of the same exact histogram."""
    other = dd.KERNEL_POPC if timed.kernel_used == dd.KERNEL_MMA else dd.KERNEL_MMA
    o = ctx.histogram(dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, k, kernel=other))
    assert o.kernel_used == other
    same = o.raw == timed.raw and o.counts == timed.counts
    assert same, "the two kernels disagree on the headline histogram"
    name = {dd.KERNEL_POPC: "popc", dd.KERNEL_MMA: "mma"}
    return {"cross_kernel": same, "timed_kernel": name[timed.kernel_used], "other_kernel": name[other],
            "other_kernel_pairs_per_s": pairs_of(k) / (o.kernel_ms * 1e-3),
            "sha256_counts": counts_digest(timed.counts)}


# ------------------------------------------------------------------------------------
# the B200 arm
# ------------------------------------------------------------------------------------
def main() -> None:
    args = parse()
    if args.impl == "reference":
        reference_arm(args)
        return
    import torch
    import coding_reliability_b200 as dd

    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import torch.distributed as dist
        from datetime import timedelta
        dist.init_process_group("nccl", timeout=timedelta(seconds=600), device_id=torch.device("cuda", local))
    stream = torch.cuda.current_stream()
    ctx = dd.Context(local, stream.cuda_stream)
    A, k = WORKLOADS[args.workload]
    kernel = {"auto": dd.KERNEL_AUTO, "popc": dd.KERNEL_POPC, "mma": dd.KERNEL_MMA}[args.kernel]
    tuning = ctx.autotune() if kernel == dd.KERNEL_AUTO else None
    if args.epilogue != "auto":
        ctx.set_mma_epilogue(dd.MMA_EPILOGUE_PAIRED if args.epilogue == "paired" else dd.MMA_EPILOGUE_SINGLE)
    launches = []  # (phase, kernel, ms): CUDA-event times, for --launch-log
    if tuning:
        for name, key in (("popc_red", "popc_red_pairs_per_s"), ("popc_ldst", "popc_ldst_pairs_per_s"),
                          ("mma_single", "mma_single_pairs_per_s"), ("mma_paired", "mma_paired_pairs_per_s")):
            launches.append(("autotune probe A=65521 k=20 (best of 2 timed, 3 run)", name,
                             tuning["probe_pairs"] / tuning[key] * 1e3))
    req = dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, k, kernel=kernel)
    P = pairs_of(k)

    def barrier():
        torch.cuda.synchronize()
        if world > 1:
            import torch.distributed as dist
            dist.barrier()
        torch.cuda.synchronize()

    def kname(r):
        return ("mma_" + dd.EPILOGUE_NAMES.get(r.mma_epilogue, "?")) if r.kernel_used == dd.KERNEL_MMA else "popc"

    for _ in range(args.warmup):
        r = ctx.histogram(req)
        launches.append((f"warm-up A={A} k={k}", kname(r), r.kernel_ms))
    popc_peak = ctx.popc_peak()  # popc/s, measured on this GPU now
    red_sweep = ctx.red_sweep()  # shared-memory atomic adds/s at 8..32 warps per SM, both table layouts
    red_best = max(red_sweep, key=lambda r: r["adds_per_s"])
    red_peak = red_best["adds_per_s"]

    clocks_dir = Path(args.clocks_dir) if args.clocks_dir else Path(tempfile.gettempdir())
    clocks = ClockSampler(local, clocks_dir / f"clocks_rank{rank}.csv")
    barrier()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    ev0.record(stream)
    kernel_ms, results = 0.0, []
    for _ in range(args.steps):
        r = ctx.histogram(req)
        kernel_ms += r.kernel_ms
        results.append(r)
    for r in results:
        launches.append((f"timed A={A} k={k}", kname(r), r.kernel_ms))
    ev1.record(stream)
    barrier()
    total_ms = ev0.elapsed_time(ev1)
    clk = clocks.stop()

    t_kernel, t_total = max_over_ranks([kernel_ms, total_ms], world, "cuda")
    # every step must produce the same exact histogram
    assert all(r.counts == results[0].counts for r in results)
    assert sum(results[0].raw) == P

    # the same histogram once more on the other kernel, outside the timed region
    parity = None
    if rank == 0 and not args.no_parity:
        parity = cross_kernel_check(ctx, dd, A, k, results[0])
        launches.append((f"parity A={A} k={k}", parity["other_kernel"], pairs_of(k) / parity["other_kernel_pairs_per_s"] * 1e3))

    value = replica_throughput(P * args.steps, world, t_kernel)
    e2e = replica_throughput(P * args.steps, world, t_total)
    per_gpu = P * args.steps / (kernel_ms * 1e-3)
    mma = results[0].kernel_used == dd.KERNEL_MMA
    if mma:
        # tcgen05 path: the tensor core computes the distances; the bound is the
        # histogram epilogue's shared-memory atomics: one per pair (single
        # epilogue) or one per two pairs (paired epilogue, packed distance pairs)
        paired = results[0].mma_epilogue == dd.MMA_EPILOGUE_PAIRED
        apr = 0.5 if paired else 1.0
        k_per_pair = MMA_K_PAD / (2 if paired else 1)  # int8 MACs per pair: one K=64 column per 2 or 1 pairs
        per_pattern = {}
        for r in red_sweep:
            per_pattern[r["pattern"]] = max(per_pattern.get(r["pattern"], 0.0), r["adds_per_s"])
        roofline = {"bound": "shared_atomic", "achieved": per_gpu * apr / 1e9, "peak": red_peak / 1e9,
                    "unit": "Gred/s", "frac": per_gpu * apr / red_peak,
                    "traffic": NCU_DRAM_BYTES_PER_LAUNCH_MMA["paired" if paired else "single"],
                    "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one mma_hist_kernel launch, "
                                      "ncu capture at k=20; operands are generated "
                                      "on chip, so the figure does not grow with k",
                    "epilogue": "paired" if paired else "single", "atomics_per_pair": apr,
                    "pairs_per_s_at_peak": red_peak / apr,
                    "peak_source": "measured live: maximum of a conflict-free red.shared.add sweep over 8..32 warps "
                                   "per SM and two table layouts (dd_measure_red_sweep); best at "
                                   f"{red_best['warps_per_sm']} warps, {red_best['pattern']}",
                    "peak_by_layout_gred_s": {k: v / 1e9 for k, v in per_pattern.items()},
                    "peak_sweep_gred_s": [[r["warps_per_sm"], r["pattern"], round(r["adds_per_s"] / 1e9, 1)]
                                          for r in red_sweep],
                    "popc_path_equivalent_frac": per_gpu / popc_peak,
                    # the tensor pipe beside it: 2 * K int8 operations per MMA column
                    "tensor_pipe": {"achieved_tops": per_gpu * 2 * k_per_pair / 1e12,
                                    "peak_tops": INT8_DENSE_TOPS_NOMINAL, "peak_source": "nominal dense int8",
                                    "frac": per_gpu * 2 * k_per_pair / 1e12 / INT8_DENSE_TOPS_NOMINAL,
                                    "ncu_tensor_cycles_active_pct": NCU_TENSOR_PIPE_PCT_MMA["paired" if paired else "single"]}}
        # and instruction issue, which bounds the epilogue
        roofline["issue"] = issue_roofline(per_gpu, "paired" if paired else "single", clk.get("sm_mhz"),
                                           torch.cuda.get_device_properties(local).multi_processor_count)
    else:
        achieved_popc = per_gpu * 1.0  # one 32-bit POPC per pair (high word folded per segment)
        roofline = {"bound": "popc", "achieved": achieved_popc / 1e9, "peak": popc_peak / 1e9, "unit": "Gpopc/s",
                    "frac": achieved_popc / popc_peak, "traffic": NCU_DRAM_BYTES_PER_LAUNCH,
                    "traffic_source": "dram__bytes_read.sum + dram__bytes_write.sum of one hist_kernel launch, "
                                      "ncu capture at k=20; the kernel reads "
                                      "only its job table and writes only its bins, so the figure does not grow with k",
                    "peak_source": "measured live: dependency-free POPC loop on this GPU (dd_measure_popc_peak)"}
    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": t_kernel / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "u64", "data": "synthetic",
        "config": {"workload": f"an_exhaustive_A{A}_k{k}", "A": A, "k": k, "codeword_bits": 40, "bins": 41,
                   "pairs": P, "parallelism": f"replicas x{world}",
                   "cold_l2": "n/a: codewords generated in registers, no HBM input"},
        "roofline": roofline,
        "e2e": {"value": e2e, "unit": UNIT, "h2d_bytes_per_step": 256, "d2h_bytes_per_step": 64 * 8 * 8},
        "gpu_launches": args.steps,
        "clocks": clk,
        "kernel_used": ("mma_" + dd.EPILOGUE_NAMES.get(results[0].mma_epilogue, "?")) if mma else "popc",
        "autotune": tuning,
    }
    if parity is not None:
        line["parity"] = parity
    if rank == 0 and not args.no_extras:
        line["super_a_sweep_k16"] = super_a_extra(ctx, dd)
        line["serving"] = serving_extra(dd)
        line["ancandidates"] = candidates_extra(ctx, popc_peak)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(A)
    ctx.close()
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank == 0 and args.launch_log:
        Path(args.launch_log).write_text(json.dumps(
            {"command": " ".join(sys.argv), "launches": [{"phase": a, "kernel": b, "ms": c} for a, b, c in launches]},
            indent=1))
    if rank == 0:
        print(json.dumps(line), flush=True)


SERVING_CLASSES = ("exhaustive", "grid", "monte_carlo")


def serving_mix(dd, count=48, seed=20261203):
    """Seeded query mix: A uniform over odd 8..16-bit values, k uniform in
    {8,12,16,20,24,32}; k<=20 exhaustive; k>=24 either the grid with stride
    2^(k-16) (m = 2^16 lattice points, so 2^k * 2^16 pairs: 2^48 at k=32) or
    Monte Carlo with 2^32..2^36 Philox-drawn pairs.  Returns (class, request)."""
    import random
    rng = random.Random(seed)
    out = []
    for i in range(count):
        A = rng.randrange(129, 1 << 16) | 1
        k = rng.choice([8, 12, 16, 20, 24, 32])
        if k <= 20:
            cls, q = "exhaustive", dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, k)
        elif rng.random() < 0.5:
            cls, q = "grid", dd.Request(dd.CODE_AN, dd.MODE_GRID_1D, A, k, m=1 << 16)  # stride 2^(k-16)
        else:
            samples = 1 << rng.randrange(32, 37)
            cls, q = "monte_carlo", dd.Request(dd.CODE_AN, dd.MODE_MONTE_CARLO, A, k, m=max(1, samples >> k),
                                               seed=i + 1)
        q.user_tag = i
        out.append((cls, q))
    return out


def percentile(sorted_values: list[float], p: float) -> float:
    """Nearest-rank percentile of an ascending list."""
    n = len(sorted_values)
    return sorted_values[min(n - 1, max(0, -(-round(p * 1000) * n // 1000) - 1))]


def serving_extra(dd, rate_per_s=16.0) -> dict:
    """p50/p99 latency (submit -> result on the host clock), aggregate and per
    query class, and aggregate pairs/s of the query server on a seeded Poisson
    stream of the serving mix."""
    import random
    import threading
    mix = serving_mix(dd)
    reqs = [q for _, q in mix]
    rng = random.Random(7)
    with dd.Server(0, round_ms=20) as s:
        # warm the server (kernel images; the server autotuned when it was created)
        s.wait(s.submit(dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, 641, 12)), 60)
        tickets = []
        t0 = time.perf_counter()

        def client():
            for q in reqs:
                tickets.append(s.submit(q))
                time.sleep(rng.expovariate(rate_per_s))

        th = threading.Thread(target=client)
        th.start()
        th.join()
        results = [s.wait(t, 900) for t in tickets]
        wall = time.perf_counter() - t0
        st = s.stats()
    assert all(code == 0 for code, _ in results)
    lat = sorted(r.total_ms for _, r in results)
    pairs = sum(r.pairs for _, r in results)
    per_class = {}
    for cls in SERVING_CLASSES:
        rows = [(q, r) for (c, q), (_, r) in zip(mix, results) if c == cls]
        if not rows:
            continue
        cl = sorted(r.total_ms for _, r in rows)
        per_class[cls] = {"queries": len(rows), "p50_ms": percentile(cl, 0.50), "p99_ms": percentile(cl, 0.99),
                          "max_ms": cl[-1], "pairs": sum(r.pairs for _, r in rows),
                          "k": sorted({q.n for q, _ in rows})}
    kernels = {r.kernel_used for _, r in results}
    return {"queries": len(reqs), "arrival_rate_per_s": rate_per_s, "p50_ms": percentile(lat, 0.50),
            "p99_ms": percentile(lat, 0.99), "per_class": per_class,
            "pairs": pairs, "pairs_per_s_wall": pairs / wall, "pairs_per_s_device": st["pairs_per_s"],
            "rounds": st["rounds"], "wall_s": wall,
            "kernels_used": sorted({dd.KERNEL_POPC: "popc", dd.KERNEL_MMA: "mma"}.get(x, str(x)) for x in kernels),
            "mix": "A odd 8-16 bit, k in {8,12,16,20,24,32}; exhaustive k<=20; k>=24 grid stride 2^(k-16) "
                   "(m=2^16) or Monte Carlo 2^32..2^36 samples"}


def super_a_set(count=256, seed=20261203):
    import random
    rng = random.Random(seed)
    out = []
    while len(out) < count:
        a = rng.randrange(32768, 65536) | 1
        if a not in out:
            out.append(a)
    return out


def super_a_extra(ctx, dd) -> dict:
    """k=16 sweep over 256 seeded odd A in [32768, 65536), three ways:
      batched_*   ONE persistent, graph-captured launch for all 256 instances;
      single_*    256 dd_histogram calls, one persistent launch per instance
                  (the reference's loop over A, super_a/src/main.cpp:247-297,
                  on this GPU's kernels);
      plain       256 dd_histogram_plain calls (the reference's kernel design:
                  one thread per row, bins allocated/copied/freed per call).
    speedup_vs_single_launch isolates batching + graph replay; speedup_vs_plain
    adds the kernel design."""
    As = super_a_set()
    reqs = [dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, 16, convention=dd.CONV_SUPER_A) for A in As]
    P = pairs_of(16) * len(As)
    out = {}
    batched = None
    for name, kernel in (("batched_popc", dd.KERNEL_POPC), ("batched_mma", dd.KERNEL_MMA)):
        for _ in range(3):
            ctx.batch(reqs, use_graph=True, kernel=kernel)
        reps = 5
        t = time.perf_counter()
        for _ in range(reps):
            res = ctx.batch(reqs, use_graph=True, kernel=kernel)
        wall = (time.perf_counter() - t) / reps
        out[name] = {"pairs_per_s": P / wall, "kernel_pairs_per_s": P / (res[0].kernel_ms * 1e-3),
                     "wall_s": wall}
        batched = batched or res
    singles = {}
    for name, kernel in (("single_popc", dd.KERNEL_POPC), ("single_mma", dd.KERNEL_MMA)):
        one = [dd.Request(dd.CODE_AN, dd.MODE_EXHAUSTIVE, A, 16, convention=dd.CONV_SUPER_A, kernel=kernel)
               for A in As]
        for q in one[:8]:
            ctx.histogram(q)
        t = time.perf_counter()
        kernel_s = 0.0
        got = []
        for q in one:
            r = ctx.histogram(q)
            kernel_s += r.kernel_ms * 1e-3
            got.append(r)
        wall = time.perf_counter() - t
        assert all(a.counts == b.counts for a, b in zip(batched, got)), f"batched != {name}"
        singles[name] = {"pairs_per_s": P / wall, "kernel_pairs_per_s": P / kernel_s, "wall_s": wall}
    for r in reqs[:8]:
        ctx.histogram_plain(r)
    t = time.perf_counter()
    plain_kernel = 0.0
    plain = []
    for r in reqs:
        x = ctx.histogram_plain(r)
        plain_kernel += x.kernel_ms * 1e-3
        plain.append(x)
    plain_wall = time.perf_counter() - t
    assert all(a.counts == b.counts for a, b in zip(batched, plain)), "batched != plain"
    best = max(out.values(), key=lambda v: v["pairs_per_s"])
    best_single = max(singles.values(), key=lambda v: v["pairs_per_s"])
    out.update(singles)
    out.update({"instances": len(As), "k": 16, "pairs": P,
                "plain_pairs_per_s": P / plain_wall, "plain_kernel_pairs_per_s": P / plain_kernel,
                "plain_wall_s": plain_wall,
                "speedup_vs_plain": plain_wall / best["wall_s"],
                "speedup_vs_single_launch": best_single["wall_s"] / best["wall_s"]})
    return out


def candidates_extra(ctx, popc_peak: float) -> dict:
    """Super-A candidate pre-filter (dd_an_candidates) over every cell with A
    width 14..17 and data width 1..24, checked against the reference tool's
    golden digests; the reference's own ANcandidates (OpenMP, all host cores)
    timed on the A-width-15 cells beside the GPU time of the same cells."""
    import hashlib
    gold = {(c["k"], c["a"]): c for c in
            json.loads((ROOT / "tests" / "golden" / "ancandidates.json").read_text())}
    cells = [(k, a) for a in range(14, 18) for k in range(1, 25)]
    ctx.an_candidates(8, 14)  # warm-up
    kernel_ms, evals, popcs, ok, a15_ms = 0.0, 0, 0, True, 0.0
    for k, a in cells:
        info, lst = ctx.an_candidates(k, a)
        kernel_ms += info["kernel_ms"]
        evals += info["evaluations"]
        popcs += info["evaluations"] * (2 if k + a + 2 > 32 else 1)
        if a == 15:
            a15_ms += info["total_ms"]
        g = gold[(k, a)]
        ok &= (info["sdr"], len(lst), hashlib.sha256(",".join(map(str, lst)).encode()).hexdigest()) == \
            (g["sdr"], g["count"], g["sha256"])
    out = {"cells": len(cells), "widths": "A 14..17 bits x data 1..24 bits", "kernel_s": kernel_ms * 1e-3,
           "evaluations": evals, "evaluations_per_s": evals / (kernel_ms * 1e-3),
           "popc_frac": popcs / (kernel_ms * 1e-3) / popc_peak, "matches_reference_golden": bool(ok),
           "gpu_a15_s": a15_ms * 1e-3}
    import oracle
    if oracle.ref_ancandidates_available():
        t = time.perf_counter()
        oracle.ref_ancandidates(15, 15, 1, 24, timeout=900)
        out["reference_cpu_a15_s"] = time.perf_counter() - t
        out["reference_cpu_cores"] = os.cpu_count()
        out["speedup_a15_vs_reference_cpu"] = out["reference_cpu_a15_s"] / out["gpu_a15_s"]
    return out


if __name__ == "__main__":
    main()

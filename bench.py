#!/usr/bin/env python
"""Benchmark of the pair-counting hot path on one or more B200s.

Workload (the clustered 3-D autocorrelation the headline metric is quoted on):
  data     1,000,000 points, Neyman-Scott: 10,000 uniform parents in the unit
           cube x 100 children with N(0, 0.005^2) isotropic offsets, wrapped
           periodically (numpy seed 11)
  randoms  20,000,000 uniform points in the unit cube (numpy seed 12)
  edges    21 radii logspace(-3, -1, 21) (20 bins)
  fields   64 jackknife fields on a 4x4x4 grid: 16*floor(4x)+4*floor(4y)+floor(4z)
Synthetic inputs of the named shapes (no dataset is involved).

A step is DD + DR + RR for all 21 edges: one kd_count_batch call on prebuilt
trees, inputs resident in HBM.  value = pairs tested per second, all ranks,
with the mixed FP32 + FP64-recheck counter; the plain FP64 counter is timed
on the same steps.  e2e = the same pairs per second through the C ABI from
host buffers: tree_construct of both catalogs (H2D of the points, node arrays
back to the host), the batched count, results read back, every step.  Also
reported: the FP64 form against a measured DGEMM peak, the all-pairs-
equivalent rate (Nd^2 + Nd Nr + Nr^2 per step over the step time) and an
FP32-pipe model of the binning (FMA lane-ops per pair from the measured
active edges per pair).

--gpus N (torchrun): every rank builds the trees and counts its 1/N share of
the batch's query blocks (kd_count_batch_shard); the per-rank counts are summed with
one all-reduce and checked against rank 0's expectations.  Total work is
fixed: scaling "strong".

--impl reference: the reference's own CPU path (oracle/_ref/libkdtree.so,
compiled from the reference sources) driven like clustering._autocorr, one
pair_count call per edge, all host threads, on a bounded seeded subset of the
queries against the full trees; rank 0 only.
"""
import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "pairs tested/s, exact counts: FP32+FP64-recheck vs plain FP64 on B200; CPU ref"
UNIT = "pairs/s"
N_DATA, N_PARENTS, SIGMA = 1_000_000, 10_000, 0.005
N_RAND = 20_000_000
N_FIELDS = 64
FLOP_PER_PAIR = 8  # 3 subtractions, 1 multiply, 2 fused multiply-adds per distance
WORKLOAD = ("3D clustered autocorr: 1M Neyman-Scott data (10k parents x 100, sigma 0.005, "
            "periodic), 20M uniform randoms, 21 edges logspace(-3,-1), 64 fields 4x4x4; "
            "a step is DD+DR+RR over all edges")


def make_workload(scale=1.0):
    nd, nr, npar = int(N_DATA * scale), int(N_RAND * scale), max(1, int(N_PARENTS * scale))
    rs = np.random.RandomState(11)
    parents = rs.rand(npar, 3)
    data = (np.repeat(parents, nd // npar + 1, axis=0)[:nd] +
            rs.normal(0.0, SIGMA, (nd, 3))) % 1.0
    rand = np.random.RandomState(12).rand(nr, 3)

    def fields(p):
        return (16 * np.floor(4 * p[:, 0]) + 4 * np.floor(4 * p[:, 1]) +
                np.floor(4 * p[:, 2])).astype(np.int32)
    radii = np.logspace(-3, -1, 21)
    return (np.ascontiguousarray(data), fields(data), np.ascontiguousarray(rand), fields(rand),
            radii)


# ----------------------------------------------------------------- helpers

class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""

    QUERY = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.proc = None
        self.path = None

    def __enter__(self):
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.QUERY}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None
        return self

    def __exit__(self, *exc):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        rows = []
        try:
            for line in open(self.path):
                f = [x.strip() for x in line.split(",")]
                if len(f) >= 9:
                    rows.append(f)
        except OSError:
            pass
        finally:
            if self.path and os.path.exists(self.path):
                os.unlink(self.path)
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[5:9]) if v == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def gemm_peak_tflops(device, dtype="float32"):
    """Measured FP32 or FP64 peak: cuBLAS SGEMM (TF32 off) or DGEMM 8192^3,
    best of 5 (the analogue of the driver's bf16 GEMM measurement)."""
    try:
        import torch
        torch.backends.cuda.matmul.allow_tf32 = False
        dev = torch.device("cuda", device)
        n = 8192
        dt = getattr(torch, dtype)
        a = torch.randn(n, n, device=dev, dtype=dt)
        b = torch.randn(n, n, device=dev, dtype=dt)
        for _ in range(2):
            torch.mm(a, b)
        torch.cuda.synchronize(dev)
        best = 1e9
        for _ in range(5):
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record()
            torch.mm(a, b)
            e.record()
            torch.cuda.synchronize(dev)
            best = min(best, s.elapsed_time(e) * 1e-3)
        del a, b
        torch.cuda.empty_cache()
        return 2.0 * n ** 3 / best / 1e12
    except Exception as exc:  # no torch / no device: report without it
        print(f"{dtype} peak measurement unavailable: {exc}", file=sys.stderr)
        return None


def sm_count(device):
    try:
        import torch
        return torch.cuda.get_device_properties(device).multi_processor_count
    except Exception:
        return None


def shard_range(n, shard, nshards):
    """[lo, hi) of shard `shard` of n items split evenly over nshards, the
    split kd_count_radii_shard and kd_count_batch_shard apply to query blocks."""
    return n * shard // nshards, n * (shard + 1) // nshards


class Dist:
    """torch.distributed plumbing (barrier, sum/max reductions) when WORLD_SIZE > 1."""

    def __init__(self, backend="nccl"):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local = int(os.environ.get("LOCAL_RANK", "0"))
        self.backend = backend
        self.dist = None
        if self.world > 1:
            import datetime

            import torch
            import torch.distributed as dist
            if backend == "nccl":
                torch.cuda.set_device(self.local)
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
            self.dist, self.torch = dist, torch

    def barrier(self):
        if self.dist:
            self.dist.barrier()

    def reduce(self, arr, op):
        if not self.dist:
            return np.asarray(arr)
        dev = f"cuda:{self.local}" if self.backend == "nccl" else "cpu"
        t = self.torch.tensor(np.asarray(arr), device=dev)
        self.dist.all_reduce(t, op=getattr(self.dist.ReduceOp, op))
        return t.cpu().numpy()

    def close(self):
        if self.dist:
            self.dist.destroy_process_group()


# ------------------------------------------------------------------ my arm

def run_mine(args):
    from corruscant_b200 import _native as N
    D = Dist()
    N.set_device(D.local)
    data, fd, rand, fr, radii = make_workload(args.scale)
    t0 = time.perf_counter()
    td = N.build_tree(data, fd, N_FIELDS)
    tr = N.build_tree(rand, fr, N_FIELDS)
    build_s = time.perf_counter() - t0
    names = ("DD", "DR", "RR")
    jobs = [(td, td), (tr, td), (tr, tr)]

    def step(mode):
        # DD, DR and RR in one device batch (kd_count_batch): one traversal
        # and one persistent tile launch over all three counts' query blocks
        outs, stats = N.count_batch(jobs, radii, mode=mode, with_stats=True, shard=D.rank,
                                    nshards=D.world)
        return dict(zip(names, outs)), stats

    def timed(mode, k, w):
        for _ in range(w):
            step(mode)
        D.barrier()
        acc = dict(dev_ms=0.0, pairs=0, launches=0, tile_launches=0, tiles_ms=0.0, rechecked=0,
                   edge_pairs=0)
        res = None
        t0 = time.perf_counter()
        for _ in range(k):
            res, s = step(mode)
            acc["dev_ms"] += s["ms_total"]
            acc["pairs"] += s["pairs_tested"]
            acc["launches"] += s["launches"]
            acc["tile_launches"] += s["tile_launches"]
            acc["tiles_ms"] += s["ms_tiles"]
            acc["rechecked"] += s["pairs_rechecked"]
            acc["edge_pairs"] += s["edge_pairs"]
        acc["wall"] = time.perf_counter() - t0
        acc["res"] = res
        D.barrier()
        return acc

    peak = gemm_peak_tflops(D.local, "float32") if D.rank == 0 else None
    peak64 = gemm_peak_tflops(D.local, "float64") if D.rank == 0 else None
    with ClockSampler(D.local) as clk:
        mixed = timed(N.KD_MODE_MIXED, args.steps, args.warmup)
    clocks = clk.summary()
    fp64 = timed(N.KD_MODE_FP64, args.steps, max(1, args.warmup // 2))

    # exactness across ranks and modes: summed shard counts must agree
    tot_m = {k: D.reduce(v, "SUM") for k, v in mixed["res"].items()}
    tot_f = {k: D.reduce(v, "SUM") for k, v in fp64["res"].items()}
    exact = all(np.array_equal(tot_m[k], tot_f[k]) for k in tot_m)

    # e2e through the C ABI from host buffers, every step
    N.destroy(td)
    N.destroy(tr)
    e2e_pairs, e2e_wall = 0, 0.0
    h2d = data.nbytes + fd.nbytes + rand.nbytes + fr.nbytes
    d2h = 0
    for it in range(1 + args.steps):
        D.barrier()
        t0 = time.perf_counter()
        a = N.build_tree(data, fd, N_FIELDS)
        b = N.build_tree(rand, fr, N_FIELDS)
        _, s = N.count_batch([(a, a), (b, a), (b, b)], radii, with_stats=True, shard=D.rank,
                             nshards=D.world)
        p = s["pairs_tested"]
        dt = time.perf_counter() - t0
        d2h = 40 * (a.memsize + b.memsize) + 3 * 8 * len(radii) * N_FIELDS * N_FIELDS
        N.destroy(a)
        N.destroy(b)
        if it > 0:  # the first iteration warms the allocator
            e2e_pairs += p
            e2e_wall += dt

    dev_s = float(D.reduce([mixed["dev_ms"] * 1e-3], "MAX")[0])
    pairs = int(D.reduce([mixed["pairs"]], "SUM")[0])
    fdev_s = float(D.reduce([fp64["dev_ms"] * 1e-3], "MAX")[0])
    fpairs = int(D.reduce([fp64["pairs"]], "SUM")[0])
    e_wall = float(D.reduce([e2e_wall], "MAX")[0])
    e_pairs = int(D.reduce([e2e_pairs], "SUM")[0])
    rechecked = int(D.reduce([mixed["rechecked"]], "SUM")[0])

    if D.rank == 0:
        value = pairs / dev_s
        # the dominant kernel: k_tiles, one launch per step (DD+DR+RR batch)
        launch_pairs = mixed["pairs"] / max(1, mixed["tile_launches"])
        launch_ms = mixed["tiles_ms"] / max(1, mixed["tile_launches"])
        achieved = launch_pairs * FLOP_PER_PAIR / (launch_ms * 1e-3) / 1e12
        roofline = {"bound": "fp32", "achieved": achieved,
                    "peak": peak, "unit": "TFLOP/s",
                    "frac": (achieved / peak) if peak else None,
                    "traffic": TILE_TRAFFIC_PER_PAIR * launch_pairs
                    if TILE_TRAFFIC_PER_PAIR else None,
                    "kernel": "k_tiles<mixed> (one launch: DD+DR+RR batch)",
                    "peak_source": "measured in this run: cuBLAS SGEMM 8192^3, TF32 off",
                    "flop_per_pair": FLOP_PER_PAIR}
        # FP32-pipe model of the binning itself: per pair 3 FMA lane-ops for
        # the distance and 3 per active edge (ramp, count, band check)
        kbar = mixed["edge_pairs"] / max(1, mixed["pairs"])
        nsm, mhz = sm_count(D.local), clocks.get("sm_mhz")
        ops = 3.0 + 3.0 * kbar
        pipe_bound = 128.0 * nsm * mhz * 1e6 / ops if (nsm and mhz) else None
        tile_rate = launch_pairs / (launch_ms * 1e-3)
        pipe_model = {"active_edges_per_pair": kbar, "fma_lane_ops_per_pair": ops,
                      "bound_pairs_per_s": pipe_bound,
                      "frac": tile_rate / pipe_bound if pipe_bound else None,
                      "basis": "128 FP32 lanes/SM/clock x SMs x median SM clock"}
        f_launch_pairs = fp64["pairs"] / max(1, fp64["tile_launches"])
        f_launch_ms = fp64["tiles_ms"] / max(1, fp64["tile_launches"])
        f_achieved = f_launch_pairs * FLOP_PER_PAIR / (f_launch_ms * 1e-3) / 1e12
        fp64_roofline = {"bound": "fp64", "achieved": f_achieved, "peak": peak64,
                         "unit": "TFLOP/s", "frac": (f_achieved / peak64) if peak64 else None,
                         "kernel": "k_tiles<fp64>",
                         "peak_source": "measured in this run: cuBLAS DGEMM 8192^3"}
        nd, nr = len(data), len(rand)
        all_pairs = float(nd) * nd + float(nr) * nd + float(nr) * nr
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": D.world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": dev_s / args.steps * 1e3, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic (seeded Neyman-Scott data and uniform randoms)",
            "config": {"workload": WORKLOAD, "n_data": len(data), "n_rand": len(rand),
                       "edges": len(radii), "fields": N_FIELDS,
                       "parallelism": f"query blocks sharded over {D.world} GPU(s)",
                       "l2": "inputs larger than L2 (20M tree points: 640 MB FP64 + 320 MB FP32)"},
            "fp64_form": {"value": fpairs / fdev_s, "ms_per_step": fdev_s / args.steps * 1e3,
                          "dtype": "f64", "roofline": fp64_roofline},
            "all_pairs_equivalent_per_s": all_pairs / (dev_s / args.steps),
            "fp32_pipe_model": pipe_model,
            "mixed_over_fp64": (pairs / dev_s) / (fpairs / fdev_s),
            "counts_exact_mixed_vs_fp64": bool(exact),
            "recheck_rate": rechecked / max(1, pairs),
            "build_s": build_s,
            "roofline": roofline,
            "e2e": {"value": e_pairs / e_wall, "unit": UNIT, "h2d_bytes_per_step": int(h2d),
                    "d2h_bytes_per_step": int(d2h), "s_per_step": e_wall / args.steps},
            "clocks": clocks,
            "gpu_launches": int(mixed["launches"]),
        }
        if D.world == 1 and not args.no_cpu_baseline:
            line["cpu_baseline"] = cpu_baseline(data, fd, rand, fr, radii,
                                                n_queries=args.cpu_queries)
        print(json.dumps(line), flush=True)
    D.close()


# Per-pair DRAM traffic of the tile kernel from an ncu capture (bytes read +
# written by k_tiles over pairs tested; profiles/k_tiles_config2.md), scaled
# to a full RR launch by its pairs.
TILE_TRAFFIC_PER_PAIR = None


# ------------------------------------------------------- reference (CPU) arm

def _ref_sample(rs, n, k):
    return np.sort(rs.choice(n, size=min(k, n), replace=False))


def cpu_baseline(data, fd, rand, fr, radii, n_queries=4000, steps=1, warmup=0):
    """The reference's pthreaded CPU path (oracle/_ref, compiled from its
    sources) on a seeded query subset of DD, DR and RR against the full
    trees, one pair_count call per edge like clustering._autocorr.  Its
    "pairs tested" are the node distance evaluations of its traversal,
    counted by the oracle over the same node arrays."""
    from oracle import oracle as O
    if not O.ref_available():
        return {"value": None, "unit": UNIT, "kind": "reference",
                "unavailable": "oracle/_ref not built (make -C oracle ref)"}
    R = O.RefLib()
    cores = os.cpu_count() or 1
    td = R.build(data, fd, N_FIELDS)
    tr = R.build(rand, fr, N_FIELDS)
    rs = np.random.RandomState(13)
    sd = _ref_sample(rs, len(data), n_queries)
    sr = _ref_sample(rs, len(rand), n_queries)
    jobs = (("DD", td, data[sd], fd[sd]), ("DR", tr, data[sd], fd[sd]),
            ("RR", tr, rand[sr], fr[sr]))
    nthreads = max(1, min(cores, n_queries // 20))  # pair_count exits above n/20
    per_type = {name: [] for name, _, _, _ in jobs}
    for it in range(warmup + steps):
        for name, t, q, qf in jobs:
            t0 = time.perf_counter()
            for r in radii:
                R.pair_count(t, q, qf, N_FIELDS, r, nthreads)
            if it >= warmup:
                per_type[name].append(time.perf_counter() - t0)
    visits = 0
    nodes = {"DD": R.nodes(td), "DR": R.nodes(tr)}
    nodes["RR"] = nodes["DR"]
    for name, _, q, _ in jobs:
        for r in radii:
            visits += O.count_visits(nodes[name], q, r, nthreads=cores)
    R.destroy(td)
    R.destroy(tr)
    tt = {k: float(np.median(v)) for k, v in per_type.items()}
    t = sum(tt.values())
    nq = {"DD": len(data), "DR": len(data), "RR": len(rand)}
    full_s = sum(tt[k] * nq[k] / n_queries for k in tt)
    return {"value": visits / t, "unit": UNIT, "cores": nthreads, "kind": "reference",
            "sample": (f"{n_queries} seeded query points each for DD, DR and RR against the full "
                       f"{len(data)}/{len(rand)}-point trees, {len(radii)} pair_count calls per "
                       f"count type"),
            "s_per_sample": t, "pairs_tested_per_sample": int(visits),
            "full_result_s_extrapolated": full_s,
            "note": "pairs tested on the CPU = reference traversal node visits"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    data, fd, rand, fr, radii = make_workload(args.scale)
    cb = cpu_baseline(data, fd, rand, fr, radii, n_queries=args.cpu_queries, steps=args.steps,
                      warmup=args.warmup)
    if cb.get("value") is None:
        print(json.dumps({"impl": "reference", "unavailable": cb.get("unavailable")}))
        return
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cb["s_per_sample"] * 1e3,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": "synthetic (seeded Neyman-Scott data and uniform randoms)",
            "config": {"workload": WORKLOAD, "n_data": len(data), "n_rand": len(rand),
                       "edges": len(radii), "fields": N_FIELDS},
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "e2e": {"value": cb["value"], "unit": UNIT, "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("mine", "reference"), default="mine")
    ap.add_argument("--scale", type=float, default=1.0, help="workload size factor (1 = full)")
    ap.add_argument("--cpu-queries", type=int, default=4000,
                    help="query points per count type in the CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "mine":
        ap.error("at least 3 warm-up steps")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_mine(args)


if __name__ == "__main__":
    main()

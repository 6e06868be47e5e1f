#!/usr/bin/env python
"""Benchmark of the pair-counting hot path on one or more B200s.

Default workload (--workload clustered3d, the clustered 3-D autocorrelation
the headline metric is quoted on):
  data     1,000,000 points, Neyman-Scott: 10,000 uniform parents in the unit
           cube x 100 children with N(0, 0.005^2) isotropic offsets, wrapped
           periodically (numpy seed 11)
  randoms  20,000,000 uniform points in the unit cube (numpy seed 12)
  edges    21 radii logspace(-3, -1, 21) (20 bins)
  fields   64 jackknife fields on a 4x4x4 grid: 16*floor(4x)+4*floor(4y)+floor(4z)
Other workloads, measured the same way (seeded synthetic inputs of the named
shapes; no dataset is involved):
  angular  2,000,000 (RA, DEC) points in RA 0-90 deg, DEC -10..60 deg uniform
           in sin DEC, half of them in Gaussian blobs (sigma 0.05 deg, tangent
           plane) around 20,000 centres; 20,000,000 uniform randoms; 16 edges
           theta = logspace(-3, log10 2, 16) deg as chords; 100 fields
           auto-divided from the data (corruscant_b200.fields: HEALPix pixels
           partitioned into balanced fields, min_ratio 0.5); DD + DR + RR
  mocks    128 Neyman-Scott catalogs (N/100 parents, sigma 0.005) with sizes
           log-uniform in 20,000..500,000, one shared 5,000,000-point uniform
           random catalog; 13 edges logspace(log10 2e-3, -1, 13); 16 fields
           4*floor(4x)+floor(4y); DD_i and D_iR for every catalog plus RR:
           257 counts in one batch
  lattice  4,000,000 data points on the 1/1024 lattice with 10% of the rows
           replaced by copies of other rows, 4,000,000 randoms on the same
           lattice; 30 edges sqrt(k)/1024 for 30 log-spaced integers k in
           [1, 10486] (many pairs exactly on an edge); 27 fields 3x3x3; both
           cross counts (DR and RD); the FP64 recheck rate is reported

A step is every count of the workload for all edges: one kd_count_batch call
on prebuilt trees, inputs resident in HBM.  value = pairs tested per second,
all ranks, with the mixed FP32 + FP64-recheck counter; the plain FP64 counter
is timed on the same steps.  e2e = a full result end to end through the C ABI
from pinned host buffers, every step: kd_tree_construct_deferred of every
catalog (two at a time; four for the 129 mock catalogs), with the H2D of the
points and, for the angular workload, the RA/DEC conversion; the batched
count while the node arrays drain to the host; the results read back and
every node array complete on the host (kd_tree_wait_nodes).  Its value is in
all-pairs-equivalent pairs per second (sum of Nq * Nt over the counts per
second of a full result), the unit the reference arm's e2e uses too, so that
their ratio is the ratio of times per full result.  Also reported: the FP64
form against its CUDA-core peak, the time per full result and an FP32-pipe
model of the binning (FMA lane-ops per pair from the measured active edges
per pair).  The default run then measures the angular, mocks and lattice
workloads at full size (a few steps each, both precisions, e2e, reference
sample) under "other_workloads".

--gpus N (torchrun): every rank builds the trees and counts its 1/N share of
the batch's query blocks (kd_count_batch_shard); the per-rank counts are
summed with one all-reduce and checked across modes.  Total work is fixed:
scaling "strong".

--impl reference: the reference's own CPU path (oracle/_ref/libkdtree.so,
compiled from the reference sources) driven like clustering._autocorr, one
pair_count call per edge, all host threads, on a bounded seeded subset of the
queries of every count against the full trees; rank 0 only.  The same leg,
run as this arm's cpu_baseline, also checks the GPU's counts for those query
subsets against the reference's.
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
# end-to-end rates of both arms: exhaustive-equivalent pairs (sum of Nq * Nt
# over the counts) per second of a full result, comparable across algorithms
E2E_UNIT = "all-pairs-equivalent pairs/s"
# catalogs built at once in the end-to-end steps: two for a few large ones
# (the smaller build, and for sky catalogs the host RA/DEC conversion, overlap
# the larger: clustered builds 81 ms against 87 ms one after the other,
# angular step 0.37 s against 0.39 s), four for many small ones (the 129 mock
# catalogs: 0.28 s against 0.62 s of builds)
E2E_BUILD_WORKERS_FEW, E2E_BUILD_WORKERS_MANY = 2, 4
FLOP_PER_PAIR = 8  # 3 subtractions, 1 multiply, 2 fused multiply-adds per distance

# ---------------------------------------------------------------- workloads


class Workload:
    """Catalogs (name -> points (n,3) f64, fields int32 or None, field count),
    counts (name, tree catalog, query catalog) and radii of one benchmark.
    radec: for catalogs given on the sky, name -> (ra, dec) in degrees, from
    which the points were computed."""

    def __init__(self, name, description, catalogs, jobs, radii, data, cpu_queries,
                 radec=None):
        self.name, self.description = name, description
        self.catalogs, self.jobs, self.radii = catalogs, jobs, np.asarray(radii, np.float64)
        self.data, self.cpu_queries, self.radec = data, cpu_queries, radec or {}


def _neyman_scott(rs, n, nparents, sigma):
    parents = rs.rand(nparents, 3)
    return (np.repeat(parents, n // nparents + 1, axis=0)[:n] +
            rs.normal(0.0, sigma, (n, 3))) % 1.0


def wl_clustered3d(scale=1.0):
    nd, nr, npar = int(1_000_000 * scale), int(20_000_000 * scale), max(1, int(10_000 * scale))
    data = _neyman_scott(np.random.RandomState(11), nd, npar, 0.005)
    rand = np.random.RandomState(12).rand(nr, 3)

    def fields(p):
        return (16 * np.floor(4 * p[:, 0]) + 4 * np.floor(4 * p[:, 1]) +
                np.floor(4 * p[:, 2])).astype(np.int32)
    return Workload(
        "clustered3d",
        ("3D clustered autocorr: 1M Neyman-Scott data (10k parents x 100, sigma 0.005, "
         "periodic), 20M uniform randoms, 21 edges logspace(-3,-1), 64 fields 4x4x4; "
         "a step is DD+DR+RR over all edges"),
        {"D": (np.ascontiguousarray(data), fields(data), 64),
         "R": (np.ascontiguousarray(rand), fields(rand), 64)},
        [("DD", "D", "D"), ("DR", "R", "D"), ("RR", "R", "R")],
        np.logspace(-3, -1, 21), "synthetic (seeded Neyman-Scott data and uniform randoms)", 4000)


def _patch_uniform(rs, n, ra_lim=(0.0, 90.0), dec_lim=(-10.0, 60.0)):
    ra = rs.uniform(ra_lim[0], ra_lim[1], n)
    s0, s1 = np.sin(np.radians(dec_lim[0])), np.sin(np.radians(dec_lim[1]))
    dec = np.degrees(np.arcsin(rs.uniform(s0, s1, n)))
    return ra, dec


def _blobs(rs, ncentres, per, sigma_deg, ra_lim=(0.0, 90.0), dec_lim=(-10.0, 60.0)):
    """Gaussian blobs in tangent-plane offsets (gnomonic projection around
    each centre); points that fall outside the patch are drawn again."""
    cra, cdec = _patch_uniform(rs, ncentres, ra_lim, dec_lim)
    a0 = np.radians(np.repeat(cra, per))
    d0 = np.radians(np.repeat(cdec, per))
    ra = np.empty(a0.size)
    dec = np.empty(a0.size)
    todo = np.arange(a0.size)
    while todo.size:
        x, y = (rs.normal(0.0, np.radians(sigma_deg), (2, todo.size)))
        rho = np.hypot(x, y)
        c = np.arctan(rho)
        rho = np.where(rho == 0, 1.0, rho)
        sd = np.cos(c) * np.sin(d0[todo]) + y * np.sin(c) * np.cos(d0[todo]) / rho
        d = np.arcsin(np.clip(sd, -1, 1))
        a = a0[todo] + np.arctan2(x * np.sin(c), rho * np.cos(d0[todo]) * np.cos(c) -
                                  y * np.sin(d0[todo]) * np.sin(c))
        a, d = np.degrees(a), np.degrees(d)
        ok = (a >= ra_lim[0]) & (a < ra_lim[1]) & (d >= dec_lim[0]) & (d < dec_lim[1])
        ra[todo[ok]], dec[todo[ok]] = a[ok], d[ok]
        todo = todo[~ok]
    return ra, dec


def wl_angular(scale=1.0):
    from corruscant_b200.twopoint import angular
    rs = np.random.RandomState(14)
    nb, nc, nr = int(1_000_000 * scale), max(1, int(20_000 * scale)), int(20_000_000 * scale)
    ra_b, dec_b = _patch_uniform(rs, nb)
    ra_c, dec_c = _blobs(rs, nc, 50, 0.05)
    ra_d, dec_d = np.concatenate([ra_b, ra_c]), np.concatenate([dec_b, dec_c])
    ra_r, dec_r = _patch_uniform(np.random.RandomState(15), nr)
    # 100 fields auto-divided from the data as the reference's fields.template
    # does it (HEALPix pixels of the data cut into balanced parts, Nside
    # doubled until the smallest field holds half the average); randoms take
    # the field of their pixel
    import contextlib
    from corruscant_b200 import fields as flds
    tpl = flds.template(100, ra=ra_d, dec=dec_d)
    with contextlib.redirect_stdout(sys.stderr):
        f_d = tpl.create_fields(min_ratio=0.5).astype(np.int32)
    f_r = tpl.assign_fields(ra=ra_r, dec=dec_r).astype(np.int32)
    theta = np.logspace(-3, np.log10(2.0), 16)
    return Workload(
        "angular",
        ("angular w(theta) autocorr: 2M (RA,DEC) points in RA 0-90, DEC -10..60 (uniform in "
         "sin DEC), half in Gaussian blobs (sigma 0.05 deg) around 20k centres; 20M uniform "
         "randoms; 16 theta edges logspace(-3,log10 2) deg as chords; 100 auto-divided fields "
         "(HEALPix pixels of the data partitioned, min_ratio 0.5); "
         "a step is DD+DR+RR over all edges"),
        {"D": (angular.cartesian(ra_d, dec_d), f_d, 100),
         "R": (angular.cartesian(ra_r, dec_r), f_r, 100)},
        [("DD", "D", "D"), ("DR", "R", "D"), ("RR", "R", "R")],
        angular.chord(theta), "synthetic (seeded sky patch: uniform + Gaussian blobs)", 4000,
        radec={"D": (ra_d, dec_d), "R": (ra_r, dec_r)})


def wl_mocks(scale=1.0):
    rs = np.random.RandomState(16)
    sizes = np.exp(rs.uniform(np.log(20_000), np.log(500_000), 128))
    sizes = np.maximum(1, (sizes * scale).astype(np.int64))

    def fields(p):
        return (4 * np.floor(4 * p[:, 0]) + np.floor(4 * p[:, 1])).astype(np.int32)
    cats, jobs = {}, []
    for i, n in enumerate(sizes):
        p = _neyman_scott(rs, int(n), max(1, int(n) // 100), 0.005)
        cats["M%03d" % i] = (np.ascontiguousarray(p), fields(p), 16)
    rand = np.random.RandomState(17).rand(int(5_000_000 * scale), 3)
    cats["R"] = (rand, fields(rand), 16)
    for i in range(len(sizes)):
        m = "M%03d" % i
        jobs.append(("DD%03d" % i, m, m))
        jobs.append(("DR%03d" % i, "R", m))
    jobs.append(("RR", "R", "R"))
    return Workload(
        "mocks",
        ("batched mocks: 128 Neyman-Scott catalogs, sizes log-uniform 20k..500k, each with "
         "its DD and its count against one shared 5M uniform random catalog, plus RR (257 "
         "counts in one batch); 13 edges logspace(log10 2e-3,-1); 16 fields 4x4 in x,y"),
        cats, jobs, np.logspace(np.log10(2e-3), -1, 13),
        "synthetic (seeded Neyman-Scott catalogs and uniform randoms)", 500)


def wl_lattice(scale=1.0):
    n = int(4_000_000 * scale)
    rs = np.random.RandomState(18)
    data = rs.randint(0, 1024, (n, 3)) / 1024.0
    dup = rs.rand(n) < 0.10
    data[dup] = data[rs.randint(0, n, int(dup.sum()))]
    rand = np.random.RandomState(19).randint(0, 1024, (n, 3)) / 1024.0

    def fields(p):
        return (9 * np.floor(3 * p[:, 0]) + 3 * np.floor(3 * p[:, 1]) +
                np.floor(3 * p[:, 2])).astype(np.int32)
    k = np.unique(np.round(np.geomspace(1, 10486, 32)).astype(np.int64))  # 30 distinct
    return Workload(
        "lattice",
        ("exactness stress cross-correlation: 4M points on the 1/1024 lattice with 10% "
         "duplicated rows, 4M lattice randoms, 30 edges sqrt(k)/1024 (k log-spaced in "
         "[1,10486]), 27 fields 3x3x3; a step is DR+RD over all edges"),
        {"D": (np.ascontiguousarray(data), fields(data), 27),
         "R": (np.ascontiguousarray(rand), fields(rand), 27)},
        [("DR", "R", "D"), ("RD", "D", "R")],
        np.sqrt(k.astype(np.float64)) / 1024.0, "synthetic (seeded lattice points)", 4000)


WORKLOADS = {"clustered3d": wl_clustered3d, "angular": wl_angular, "mocks": wl_mocks,
             "lattice": wl_lattice}


def make_workload(scale=1.0):
    """The default workload as (data, data fields, randoms, random fields, radii)."""
    w = wl_clustered3d(scale)
    (d, fd, _), (r, fr, _) = w.catalogs["D"], w.catalogs["R"]
    return d, fd, r, fr, w.radii


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


SHARD_CHUNK = 32  # blocks per interleaved chunk, as the library splits query blocks


def shard_items(n, shard, nshards, chunk=SHARD_CHUNK):
    """Indices of shard `shard` of n items split over nshards the way
    kd_count_radii_shard and kd_count_batch_shard split query blocks:
    interleaved chunks of `chunk` items, chunk c to shard c mod nshards."""
    idx = np.arange(n)
    return idx[(idx // chunk) % nshards == shard]


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
            # short, so that a rank that died ends the others' next
            # collective with an error; long enough for the slowest gap
            # between collectives: every rank generating the 20M-point
            # workload on shared host cores before the first one
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=300))
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

def _build_all(N, w, convert=False, host=None, deferred=False, workers=1):
    """Trees of every catalog; with convert, sky catalogs are converted from
    RA/DEC on the host first (the e2e path); host: the inputs to use instead
    of the workload's own arrays (pinned copies); deferred: builds that
    return before their node arrays reach the host (N.wait_nodes waits);
    workers > 1: that many catalogs built at once from host threads (each
    build runs on its own stream and releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor

    from corruscant_b200.twopoint import angular

    def one(item):
        name, (pts, f, nf) = item
        if host is not None:
            pts, f = host[name][0], host[name][1]
        if convert and name in w.radec:
            src = host[name][2] if host is not None else w.radec[name]
            pts = angular.cartesian(*src)
        return name, N.build_tree(pts, f, nf, deferred=deferred)

    # the largest catalogs first, so the small ones fill in beside them
    items = sorted(w.catalogs.items(), key=lambda kv: -len(kv[1][0]))
    if workers <= 1 or len(items) == 1:
        return dict(map(one, items))
    with ThreadPoolExecutor(max_workers=workers) as ex:
        return dict(ex.map(one, items))


def _e2e_workers(w):
    return E2E_BUILD_WORKERS_MANY if len(w.catalogs) > 4 else E2E_BUILD_WORKERS_FEW


def _pinned_copies(w):
    """Page-locked copies of every input array (points, fields, RA/DEC), the
    host buffers the end-to-end steps copy to the device from.  The torch
    tensors that own the memory are returned with the views."""
    try:
        import torch
    except ImportError:
        return None, []
    keep, host = [], {}

    def pin(a):
        if a is None:
            return None
        t = torch.empty(a.shape, dtype=getattr(torch, str(a.dtype))).pin_memory()
        v = t.numpy()
        v[...] = a
        keep.append(t)
        return v
    try:
        for name, (pts, f, _) in w.catalogs.items():
            rd = w.radec.get(name)
            host[name] = (pin(pts), pin(f), None if rd is None else (pin(rd[0]), pin(rd[1])))
    except RuntimeError as exc:  # no driver to pin with: the arrays stay pageable
        print(f"pinned host buffers unavailable: {exc}", file=sys.stderr)
        return None, []
    return host, keep


def _all_pairs(w):
    """Sum over the workload's counts of Nq * Nt (raw catalog sizes): the
    pairs an exhaustive count would test, a unit that does not depend on the
    algorithm (the reference and this engine test different pair sets)."""
    sizes = {k: len(v[0]) for k, v in w.catalogs.items()}
    return float(sum(sizes[q] * sizes[t] for _, t, q in w.jobs))


def _measure(N, D, w, steps, warmup):
    """Time one workload: `steps` device-timed steps per precision after
    `warmup` untimed ones (inputs resident in HBM), then `steps` end-to-end
    steps from pinned host buffers.  Returns the raw figures, reduced over
    ranks (device times: max; pairs: sum)."""
    radii = w.radii
    t0 = time.perf_counter()
    trees = _build_all(N, w)
    build_s = time.perf_counter() - t0
    names = [j for j, _, _ in w.jobs]
    jobs = [(trees[t], trees[q]) for _, t, q in w.jobs]

    def step(mode):
        # every count of the workload in one device batch (kd_count_batch):
        # one traversal and one persistent tile launch over all their blocks
        outs, stats = N.count_batch(jobs, radii, mode=mode, with_stats=True, shard=D.rank,
                                    nshards=D.world)
        return dict(zip(names, outs)), stats

    def timed(mode, k, wu):
        for _ in range(wu):
            step(mode)
        D.barrier()
        acc = dict(dev_ms=0.0, pairs=0, launches=0, tile_launches=0, tiles_ms=0.0, rechecked=0,
                   edge_pairs=0, accepted=0, one_bin_multifield=0, trav_ms=0.0)
        res = None
        for _ in range(k):
            res, s = step(mode)
            acc["dev_ms"] += s["ms_total"]
            acc["pairs"] += s["pairs_tested"]
            acc["launches"] += s["launches"]
            acc["tile_launches"] += s["tile_launches"]
            acc["tiles_ms"] += s["ms_tiles"]
            acc["rechecked"] += s["pairs_rechecked"]
            acc["edge_pairs"] += s["edge_pairs"]
            acc["accepted"] += s["pairs_accepted"]
            acc["one_bin_multifield"] += s["pairs_one_bin_multifield"]
            acc["trav_ms"] += s["ms_traverse"]
        acc["res"] = res
        D.barrier()
        return acc

    with ClockSampler(D.local) as clk:
        mixed = timed(N.KD_MODE_MIXED, steps, warmup)
    clocks = clk.summary()
    fp64 = timed(N.KD_MODE_FP64, steps, max(1, warmup // 2))

    # exactness across ranks and modes: summed shard counts must agree
    tot_m = {k: D.reduce(v, "SUM") for k, v in mixed["res"].items()}
    tot_f = {k: D.reduce(v, "SUM") for k, v in fp64["res"].items()}
    exact = all(np.array_equal(tot_m[k], tot_f[k]) for k in tot_m)

    # e2e through the C ABI from pinned host buffers, every step: tree
    # builds (H2D of the points, the RA/DEC conversion for sky catalogs), the
    # batched count while the node arrays drain to the host, results and
    # every node array on the host
    for t in trees.values():
        N.destroy(t)
    host, _keep = _pinned_copies(w)
    e2e_pairs, e2e_wall = 0, 0.0
    h2d = 0
    for name, (pts, f, _) in w.catalogs.items():
        h2d += (2 * 8 * len(pts) if name in w.radec else pts.nbytes) + (f.nbytes if f is not None else 0)
    d2h = 0
    for it in range(1 + steps):
        D.barrier()
        t0 = time.perf_counter()
        tt = _build_all(N, w, convert=True, host=host, deferred=True, workers=_e2e_workers(w))
        _, s = N.count_batch([(tt[t], tt[q]) for _, t, q in w.jobs], radii, with_stats=True,
                             shard=D.rank, nshards=D.world)
        for t in tt.values():  # every node array complete on the host
            N.wait_nodes(t)
        dt = time.perf_counter() - t0
        d2h = 40 * sum(t.memsize for t in tt.values()) + 8 * len(radii) * sum(
            tt[t].num_fields * tt[q].num_fields for _, t, q in w.jobs)
        if len(tt) <= 4:  # where the builds of the last step spent their time
            bstats = {k: {f: round(v, 3) if isinstance(v, float) else v
                          for f, v in N.build_stats(t).items()} for k, t in tt.items()}
        else:
            bstats = {"catalogs": len(tt), "ms_total_host_sum": round(sum(
                N.build_stats(t)["ms_total_host"] for t in tt.values()), 3)}
        count_s = s["ms_total"] * 1e-3
        for t in tt.values():
            N.destroy(t)
        if it > 0:  # the first iteration warms the allocator
            e2e_pairs += s["pairs_tested"]
            e2e_wall += dt
    del _keep
    return dict(
        build_s=build_s, clocks=clocks, exact=bool(exact), mixed=mixed, fp64=fp64,
        dev_s=float(D.reduce([mixed["dev_ms"] * 1e-3], "MAX")[0]),
        pairs=int(D.reduce([mixed["pairs"]], "SUM")[0]),
        fdev_s=float(D.reduce([fp64["dev_ms"] * 1e-3], "MAX")[0]),
        fpairs=int(D.reduce([fp64["pairs"]], "SUM")[0]),
        e_wall=float(D.reduce([e2e_wall], "MAX")[0]),
        e_pairs=int(D.reduce([e2e_pairs], "SUM")[0]),
        rechecked=int(D.reduce([mixed["rechecked"]], "SUM")[0]),
        h2d=int(h2d), d2h=int(d2h), pinned=host is not None, build_stats=bstats,
        e2e_count_s=count_s)


def _fp64_lane_peak(device, mhz):
    """FP64 CUDA-core peak at the sampled clock: SMs x 64 FP64 lanes x 2
    FLOP (FMA) per clock.  The FP64 tiles run on that pipe, not on the FP64
    tensor cores a DGEMM uses."""
    nsm = sm_count(device)
    return nsm * 64 * 2 * mhz * 1e6 / 1e12 if (nsm and mhz) else None


def _summary(w, m, steps, peak, peak64, D):
    """The figures of one measured workload (rank 0)."""
    value = m["pairs"] / m["dev_s"]
    all_pairs = _all_pairs(w)
    s_full = m["dev_s"] / steps
    e_s = m["e_wall"] / steps
    mixed, fp64 = m["mixed"], m["fp64"]
    # the dominant kernel: k_tiles, one launch per step (the whole batch)
    launch_pairs = mixed["pairs"] / max(1, mixed["tile_launches"])
    launch_ms = mixed["tiles_ms"] / max(1, mixed["tile_launches"])
    achieved = launch_pairs * FLOP_PER_PAIR / (launch_ms * 1e-3) / 1e12
    mhz = m["clocks"].get("sm_mhz")
    nsm = sm_count(D.local)
    lane32 = nsm * 128 * 2 * mhz * 1e6 / 1e12 if (nsm and mhz) else None
    roofline = {"bound": "fp32", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
                "frac": (achieved / peak) if peak else None,
                "traffic": TILE_TRAFFIC_PER_PAIR * launch_pairs if TILE_TRAFFIC_PER_PAIR else None,
                "kernel": "k_tiles<mixed> (one launch: the step's whole batch)",
                "peak_source": "measured in this run: cuBLAS SGEMM 8192^3, TF32 off",
                "lane_peak": lane32,
                "frac_of_lane_peak": (achieved / lane32) if lane32 else None,
                "lane_peak_basis": "SMs x 128 FP32 lanes x 2 FLOP x median SM clock",
                "flop_per_pair": FLOP_PER_PAIR}
    if TILE_TRAFFIC_PER_PAIR:
        roofline["traffic_source"] = TILE_TRAFFIC_SOURCE
    # FP32-pipe model of the binning itself: per pair 3 FMA lane-ops for
    # the distance and 3 per active edge (ramp, count, band check)
    kbar = mixed["edge_pairs"] / max(1, mixed["pairs"])
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
    lane64 = _fp64_lane_peak(D.local, mhz)
    fp64_roofline = {"bound": "fp64", "achieved": f_achieved, "peak": lane64,
                     "unit": "TFLOP/s", "frac": (f_achieved / lane64) if lane64 else None,
                     "kernel": "k_tiles<fp64>",
                     "peak_source": "SMs x 64 FP64 lanes x 2 FLOP x median SM clock "
                                    "(the FP64 CUDA-core pipe the kernel runs on)",
                     "dgemm_measured": peak64}
    return {
        "value": value, "ms_per_step": s_full * 1e3, "s_per_full_result": s_full,
        "fp64_form": {"value": m["fpairs"] / m["fdev_s"],
                      "ms_per_step": m["fdev_s"] / steps * 1e3,
                      "s_per_full_result": m["fdev_s"] / steps, "dtype": "f64",
                      "roofline": fp64_roofline},
        "all_pairs_equivalent_per_s": all_pairs / s_full,
        "fp32_pipe_model": pipe_model,
        "mixed_over_fp64": value / (m["fpairs"] / m["fdev_s"]),
        "counts_exact_mixed_vs_fp64": m["exact"],
        "recheck_rate": m["rechecked"] / max(1, m["pairs"]),
        # whole node pairs inside one bin: accepted without distances (single
        # field on both sides), and those tiled only because a side holds
        # several fields
        "node_pair_accepts_per_step": {
            "pairs_accepted": mixed["accepted"] / steps,
            "pairs_one_bin_multifield": mixed["one_bin_multifield"] / steps,
            "pairs_tested": mixed["pairs"] / steps},
        "traverse_ms_per_step": mixed["trav_ms"] / steps,
        "pairs_rechecked_per_step": m["rechecked"] / steps,
        "build_s": m["build_s"],
        "roofline": roofline,
        "e2e": {"value": all_pairs / e_s, "unit": E2E_UNIT,
                "h2d_bytes_per_step": m["h2d"], "d2h_bytes_per_step": m["d2h"],
                "s_per_step": e_s, "s_per_full_result": e_s,
                "pairs_tested_per_s": m["e_pairs"] / m["e_wall"],
                "host_buffers": "pinned" if m["pinned"] else "pageable",
                "builds": (f"kd_tree_construct_deferred, {_e2e_workers(w)} catalog(s) at a time; "
                           "node arrays complete on the host before the step ends"),
                "count_device_s_last_step": m["e2e_count_s"],
                "build_stats_last_step": m["build_stats"]},
        "clocks": m["clocks"],
        "gpu_launches": int(mixed["launches"]),
    }


def _config(w, world):
    """The workload description both arms print (identical for the same
    workload and rank count)."""
    sizes = {k: len(v[0]) for k, v in w.catalogs.items()}
    cfg = {"workload": w.description, "counts": len(w.jobs), "edges": len(w.radii),
           "parallelism": f"{world} rank(s): query blocks sharded over the GPUs",
           "l2": "inputs larger than L2 (tree points stream from HBM each step)"}
    if len(sizes) <= 4:
        cfg["catalogs"] = sizes
    else:
        cfg["catalog_points_total"] = int(sum(sizes.values()))
        cfg["catalogs"] = len(sizes)
    return cfg


# the other workloads, measured by the default run after the headline one
OTHER_WORKLOADS = ("angular", "mocks", "lattice")
OTHER_STEPS = 3


def run_mine(args):
    from corruscant_b200 import _native as N
    D = Dist()
    N.set_device(D.local)
    w = WORKLOADS[args.workload](args.scale)
    peak = gemm_peak_tflops(D.local, "float32") if D.rank == 0 else None
    peak64 = gemm_peak_tflops(D.local, "float64") if D.rank == 0 else None
    m = _measure(N, D, w, args.steps, args.warmup)
    if D.rank == 0:
        line = {"metric": METRIC, "unit": UNIT, "n_gpus": D.world, "steps": args.steps,
                "warmup": args.warmup, "higher_is_better": True, "scaling": "strong",
                "vs_baseline": None, "dtype": "f32+f64", "data": w.data,
                "config": _config(w, D.world)}
        line.update(_summary(w, m, args.steps, peak, peak64, D))
        line = {k: line[k] for k in ("metric", "value", "unit", "n_gpus", "steps", "warmup",
                                     "ms_per_step")} | line
        if D.world == 1 and not args.no_cpu_baseline:
            cb = cpu_baseline(w, n_queries=args.cpu_queries, gpu=N)
            line["cpu_baseline"] = cb
            if cb.get("full_result_s_extrapolated"):
                line["speedup_per_full_result"] = {
                    "device": cb["full_result_s_extrapolated"] / line["s_per_full_result"],
                    "e2e": cb["full_result_s_extrapolated"] / line["e2e"]["s_per_full_result"]}
    # the other workloads at full size (one GPU, default workload only): a
    # few steps each, both precisions, e2e and the reference sample
    others = {}
    if D.world == 1 and args.workload == "clustered3d" and args.scale == 1.0 and not args.headline_only:
        del m
        for name in OTHER_WORKLOADS:
            wo = WORKLOADS[name](1.0)
            mo = _measure(N, D, wo, OTHER_STEPS, 3)
            o = _summary(wo, mo, OTHER_STEPS, peak, peak64, D)
            o = {"config": _config(wo, D.world), "steps": OTHER_STEPS, "warmup": 3} | {
                k: o[k] for k in ("value", "ms_per_step", "s_per_full_result", "fp64_form",
                                  "mixed_over_fp64", "counts_exact_mixed_vs_fp64", "recheck_rate",
                                  "all_pairs_equivalent_per_s", "roofline", "fp32_pipe_model",
                                  "node_pair_accepts_per_step", "e2e", "clocks", "build_s")}
            if not args.no_cpu_baseline:
                cb = cpu_baseline(wo, n_queries=args.cpu_queries, gpu=N)
                o["cpu_baseline"] = cb
                if cb.get("full_result_s_extrapolated"):
                    o["speedup_per_full_result"] = {
                        "device": cb["full_result_s_extrapolated"] / o["s_per_full_result"],
                        "e2e": cb["full_result_s_extrapolated"] / o["e2e"]["s_per_full_result"]}
            others[name] = o
            del wo, mo
    if D.rank == 0:
        if others:
            line["other_workloads"] = others
        print(json.dumps(line), flush=True)
    D.close()


# Per-pair DRAM traffic of the tile kernel (dram bytes read + written by one
# k_tiles launch over the pairs it tested), from the ncu capture of the
# clustered workload at scale 0.3 summarised in profiles/, scaled to a full
# launch by its pairs: the traffic is mostly the tile records, whose number
# grows with the pairs.
TILE_TRAFFIC_PER_PAIR = (3.271633e9 + 11.673856e6) / 2.02520e11  # bytes per pair tested
TILE_TRAFFIC_SOURCE = ("ncu dram__bytes_read.sum + dram__bytes_write.sum of one k_tiles launch, "
                       "clustered workload at scale 0.3 (2.025e11 pairs), scaled by pairs")


# ------------------------------------------------------- reference (CPU) arm

def cpu_baseline(w, n_queries=None, steps=1, warmup=0, gpu=None):
    """The reference's pthreaded CPU path (oracle/_ref, compiled from its
    sources) on a seeded query subset of every count against the full trees,
    one pair_count call per edge like clustering._autocorr.  Its "pairs
    tested" are the node distance evaluations of its traversal, counted by
    the oracle over the same node arrays.  With gpu (the corruscant_b200
    native module) the GPU's counts for the same query subsets are compared
    with the reference's."""
    from oracle import oracle as O
    if not O.ref_available():
        return {"value": None, "unit": UNIT, "kind": "reference",
                "unavailable": "oracle/_ref not built (make -C oracle ref)"}
    R = O.RefLib()
    cores = os.cpu_count() or 1
    nq_max = n_queries or w.cpu_queries
    # the reference converts sky catalogs with its own coordinate library
    pts = {}
    coords_equal = True
    for name, (p, _, _) in w.catalogs.items():
        if name in w.radec:
            pts[name] = R.radec2cart64(*w.radec[name])
            coords_equal &= bool(np.array_equal(pts[name].view(np.int64), p.view(np.int64)))
        else:
            pts[name] = p
    used = sorted({t for _, t, _ in w.jobs})
    rtrees = {n: R.build(pts[n], w.catalogs[n][1], w.catalogs[n][2]) for n in used}
    rs = np.random.RandomState(13)
    samples, skipped = [], []
    for name, t, q in w.jobs:
        n = len(pts[q])
        if n < 20:  # the reference's pair_count exits below 20 query points (kdquery.c:176)
            skipped.append(name)
            continue
        idx = np.sort(rs.choice(n, size=min(nq_max, n), replace=False))
        f = w.catalogs[q][1]
        samples.append((name, t, q, pts[q][idx], None if f is None else f[idx]))
    times = [[] for _ in samples]
    counts = [None] * len(samples)
    for it in range(warmup + steps):
        for j, (name, t, q, qp, qf) in enumerate(samples):
            nthreads = max(1, min(cores, len(qp) // 20))  # pair_count exits above n/20
            t0 = time.perf_counter()
            out = [R.pair_count(rtrees[t], qp, qf, w.catalogs[q][2], r, nthreads)
                   for r in w.radii]
            if it >= warmup:
                times[j].append(time.perf_counter() - t0)
            counts[j] = np.stack(out)
    nodes = {n: R.nodes(rtrees[n]) for n in used}
    visits = 0
    for name, t, q, qp, qf in samples:
        for r in w.radii:
            visits += O.count_visits(nodes[t], qp, r, nthreads=cores)
    parity = None
    if gpu is not None:
        gt = {n: gpu.build_tree(w.catalogs[n][0], w.catalogs[n][1], w.catalogs[n][2])
              for n in used}
        parity = True
        for (name, t, q, qp, qf), want in zip(samples, counts):
            got = gpu.count_points(gt[t], qp, qf, w.catalogs[q][2], w.radii)
            parity &= bool(np.array_equal(got, want))
        for tr in gt.values():
            gpu.destroy(tr)
    for tr in rtrees.values():
        R.destroy(tr)
    tt = [float(np.median(v)) for v in times]
    t_all = sum(tt)
    full_s = sum(tj * len(pts[q]) / len(qp) for tj, (_, _, q, qp, _) in zip(tt, samples))
    nsamp = sorted({len(s[3]) for s in samples})
    res = {"value": visits / t_all, "unit": UNIT,
           "cores": max(1, min(cores, nq_max // 20)), "kind": "reference",
           "sample": (f"{'/'.join(map(str, nsamp))} seeded query points for each of the "
                      f"{len(samples)} counts against the full trees, {len(w.radii)} "
                      f"pair_count calls per count; the sample is sized for 10-30 s of "
                      f"CPU work (a 1% query subset would take minutes per count), and "
                      f"the time per full result is extrapolated linearly in the queries"),
           "s_per_sample": t_all, "pairs_tested_per_sample": int(visits),
           "full_result_s_extrapolated": full_s,
           "note": "pairs tested on the CPU = reference traversal node visits"}
    if skipped:
        res["counts_skipped"] = skipped
    if w.radec:
        res["coordinates_bit_identical"] = coords_equal
    if parity is not None:
        res["gpu_counts_equal_reference_on_sample"] = parity
    return res


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    w = WORKLOADS[args.workload](args.scale)
    cb = cpu_baseline(w, n_queries=args.cpu_queries, steps=args.steps, warmup=args.warmup)
    if cb.get("value") is None:
        print(json.dumps({"impl": "reference", "unavailable": cb.get("unavailable")}))
        return
    cfg = _config(w, int(os.environ.get("WORLD_SIZE", "1")))
    full_s = cb["full_result_s_extrapolated"]
    line = {"impl": "reference", "metric": METRIC, "value": cb["value"], "unit": UNIT,
            "n_gpus": int(os.environ.get("WORLD_SIZE", "1")), "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": cb["s_per_sample"] * 1e3,
            "higher_is_better": True, "scaling": "strong", "vs_baseline": None,
            "dtype": "f64", "data": w.data, "config": cfg,
            "cpu_baseline": {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample")},
            "s_per_full_result": full_s,
            "full_result_s_extrapolated": full_s,
            "all_pairs_equivalent_per_s": _all_pairs(w) / full_s,
            # end to end: a full result's exhaustive-equivalent pairs per
            # second of (extrapolated) CPU time, the unit of the GPU arm's e2e
            "e2e": {"value": _all_pairs(w) / full_s, "unit": E2E_UNIT,
                    "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0,
                    "s_per_full_result": full_s}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser(description=__doc__.split("\n\n")[0])
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=("mine", "reference"), default="mine")
    ap.add_argument("--workload", choices=sorted(WORKLOADS), default="clustered3d")
    ap.add_argument("--scale", type=float, default=1.0, help="workload size factor (1 = full)")
    ap.add_argument("--cpu-queries", type=int, default=None,
                    help="query points per count in the CPU sample (default per workload)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--headline-only", action="store_true",
                    help="skip the other workloads after the default one")
    args = ap.parse_args()
    if args.warmup < 3 and args.impl == "mine":
        ap.error("at least 3 warm-up steps")
    if args.impl == "reference":
        run_reference(args)
    else:
        run_mine(args)


if __name__ == "__main__":
    main()

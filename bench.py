#!/usr/bin/env python
"""Benchmark of the SpTC path: matched products per second on one B200 (or N).

Workload: the large-output ESC contraction -- X is 2482x2862x14036x17 with
3.1M nonzeros, Zipf(s=1.1) indices per mode, U[0,1) values, seed 1; Z = X
contracted with itself on modes 2,3 (the reference CLI's ``-c 2 -x 2 3 -y 2 3``).
It has 1.749e10 matched products and 1.316e10 output nonzeros (158 GB of
output), so Z streams through HBM in chunks.  Inputs are synthetic (seeded,
same shape / distributions as the named workload).

One step = one full contraction (linearise, sort, match, symbolic + numeric
accumulation of every output chunk).  ``value``: operands resident in HBM,
output chunks produced in HBM and dropped (the reference also drops Z).
``e2e``: the same through the public API from pinned host COO buffers, with
the host->device copy of the inputs and the device->host copy of every output
chunk (into a pinned ring) inside the timed region.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --impl reference --reference-gpu   # the reference GSPARC itself on the GPU

Under torchrun the one contraction is split into row shards of about equal
matched-product mass, one per rank (the reference's multi-GPU mode): strong
scaling, operands replicated, no collective on the data path; only the time
(max over ranks) and the product counts are reduced.

``roofline``: the algorithmic bytes of the contraction (the ESC formula:
operands read and packed, the match, every matched product written and read
once, the output written once) over the contraction's CUDA-event time;
``roofline_bytes_moved``: the bytes this engine does move (it never writes a
product to HBM) over the numeric kernels' time.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import shutil
import subprocess
import sys
import tempfile
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

WORKLOAD = "esc_large"
METRIC = "matched products/sec"
UNIT = "products/s"
# ncu DRAM bytes (read + write) of the numeric launches (k_light<1>, k_rowwin<1>, k_stream) per output
# nonzero, the kept bitmaps' reads left out, measured on esc_large at scale 0.1 (one output chunk,
# 2.50e8 outputs: 307.70 MB read of which 268.27 MB kept bitmaps, 2858.71 MB written)
TRAFFIC_NUMERIC_PER_OUTPUT = 2898.144436e6 / 2.50473870e8
# kept heavy-row bitmaps: written by the symbolic pass (208.30 MB reach DRAM), read once by the numeric
# pass (268.27 MB), per kept byte, same capture
TRAFFIC_PER_KEPT_BITMAP_BYTE = 476.565904e6 / 268267904
# ncu DRAM bytes of every other kernel of a contraction (linearise, sort, match, planning, spans,
# symbolic pass reads) per operand nonzero (X + Y), same capture (310k + 310k operand nonzeros:
# 144.67 MB read; their writes stay in L2 at that size)
TRAFFIC_OTHER_PER_OPERAND_NNZ = 144.665904e6 / 620000


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--scale", type=float, default=1.0, help="nnz scale of the workload (1.0 = full)")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="target CPU work per baseline sample")
    ap.add_argument("--no-mixed", action="store_true", help="skip the mixed-stream (batched / served) lines")
    ap.add_argument("--mixed-count", type=int, default=256, help="instances of the batched / served streams")
    ap.add_argument("--served-max-nnz", type=float, default=2e6,
                    help="largest operand nnz of the served stream (the served workload's range reaches 5e7; "
                         "the default keeps the default run within minutes)")
    ap.add_argument("--served-only", action="store_true", help="run only the served stream (with its plain form)")
    ap.add_argument("--reference-gpu", action="store_true",
                    help="with --impl reference: time the reference GSPARC program itself on the GPU, and our "
                         "CLI on the same files, for the plain, ESC and dense-accumulator workloads")
    return ap.parse_args()


# --------------------------------------------------------------------------- helpers
class Clocks:
    """Samples SM clocks and throttle reasons with nvidia-smi while running."""

    Q = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        """Starts sampling and returns once the first sample is written: the
        sampler's start-up stalls the GPU for tens of milliseconds (measured:
        34 ms on the first kernel after it starts), which must not fall into
        the timed region."""
        fd, self.path = tempfile.mkstemp(suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except FileNotFoundError:
            self.proc = None
            return
        t0 = time.time()
        while time.time() - t0 < 10 and self.proc.poll() is None:
            if os.path.getsize(self.path) > 0:
                break
            time.sleep(0.05)
        time.sleep(0.5)

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons, power = [], [], set(), []
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                smax.append(float(f[1]))
                power.append(float(f[2]))
            except ValueError:
                continue
            for n, v in zip(names, f[4:8]):
                if v.lower() == "active":
                    reasons.add(n)
        os.unlink(self.path)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": max(smax), "reasons": sorted(reasons),
                "samples": len(sm), "power_w_max": max(power) if power else None}


def load_peaks() -> dict:
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return {"hbm_gbs": float(d["hbm_gbs"]), "source": "measured"}
    return {"hbm_gbs": 6650.0, "source": "fallback"}


def synth_module():
    """gsparc_b200/synth.py (numpy only), loaded from its file so that the
    reference arm never imports the package (which loads the engine library)."""
    import importlib.util
    name = "gsparc_b200_synth_standalone"
    if name not in sys.modules:
        spec = importlib.util.spec_from_file_location(name, os.path.join(ROOT, "gsparc_b200", "synth.py"))
        mod = importlib.util.module_from_spec(spec)
        sys.modules[name] = mod
        spec.loader.exec_module(mod)
    return sys.modules[name]


def workload(rank: int, scale: float):
    return synth_module().esc_large(scale=scale, seed=1 + rank)


def alg_bytes_contraction(nnz_x: int, order_x: int, nnz_y: int, order_y: int, ir: int, nnz_z: int) -> float:
    """Algorithmic bytes of one ESC contraction: read the SoA COO operands and
    write + read their packed (key, value) once, the X match (pos, cnt), the Y
    segment scan, every matched product materialised once (write + read, 12 B
    each) and the output written once."""
    b = 0.0
    for n, o in ((nnz_x, order_x), (nnz_y, order_y)):
        b += n * (8.0 * o + 4.0) + 2.0 * 12.0 * n
    return b + 16.0 * nnz_x + 8.0 * nnz_y + 24.0 * ir + 12.0 * nnz_z


def cpu_sample(X, target_products: float, seed: int = 0):
    """Rows of X (whole output rows) whose products sum to about target, plus the
    nonzero at the largest coordinate so the sample's inferred dims match Y's."""
    fx = (X.idx[0] << np.uint64(12)) | X.idx[1]
    rows, inv = np.unique(fx, return_inverse=True)
    ck = (X.idx[2] << np.uint64(5)) | X.idx[3]
    _, ci, cnt = np.unique(ck, return_inverse=True, return_counts=True)
    prod = cnt[ci].astype(np.float64)
    rp = np.bincount(inv, weights=prod)
    perm = np.random.default_rng(seed).permutation(rows.shape[0])
    k = int(np.searchsorted(np.cumsum(rp[perm]), target_products)) + 1
    take = np.zeros(rows.shape[0], bool)
    take[perm[:k]] = True
    m = take[inv]
    m[0] = True  # planted max coordinate
    return X.subset(m), int(prod[m].sum())


def run_sparta(xs_path, y_path, threads, timeout=600):
    """One run of the reference's CPU SpTC (baselines/Sparta ttt, mode 3).
    Returns its own [Total time] in seconds, or None if it failed (retried a
    few times)."""
    ttt = os.path.join(ROOT, "oracle", "_ref", "ttt")
    if not os.path.exists(ttt):
        return None
    env = dict(os.environ, EXPERIMENT_MODES="3")
    cmd = [ttt, "-X", xs_path, "-Y", y_path, "-m", "2", "-x", "2", "3", "-y", "2", "3", "-t", str(threads)]
    for _ in range(3):
        try:
            r = subprocess.run(cmd, env=env, capture_output=True, text=True, timeout=timeout)
        except subprocess.TimeoutExpired:
            continue
        for line in r.stderr.splitlines():
            if line.startswith("[Total time]"):
                return float(line.split(":")[1].split()[0])
    return None


class CpuBaseline:
    """The reference's CPU SpTC (or the oracle port) on bounded samples of the workload.
    Uses numpy and the baseline binary only: the engine library is not loaded."""

    def __init__(self, X, target_seconds: float):
        synth = synth_module()
        self.X = X
        # the cores this process may run on (the host may have more than the job is given)
        self.threads = len(os.sched_getaffinity(0)) or 1
        self.dir = tempfile.mkdtemp(prefix="gsparc_cpu_")
        self.y_path = os.path.join(self.dir, "y.tns")
        synth.write_tns(self.y_path, X)
        # calibrate on a small sample
        self.kind = "reference"
        xs, ir = cpu_sample(X, 5e6, seed=7)
        p = os.path.join(self.dir, "xs_cal.tns")
        synth.write_tns(p, xs)
        t = run_sparta(p, self.y_path, self.threads)
        if t is None or t <= 0:
            self.kind = "port"
            t = self._port_time(xs)
        rate = ir / max(t, 1e-6)
        target = min(max(rate * target_seconds, 5e6), 2e9)
        self.xs, self.ir = cpu_sample(X, target, seed=11)
        self.xs_path = os.path.join(self.dir, "xs.tns")
        synth.write_tns(self.xs_path, self.xs)
        if self.kind == "port":
            self.threads = 1

    def _port_time(self, xs):
        sys.path.insert(0, os.path.join(ROOT, "tests"))
        import oracle_bind as ob
        t0 = time.perf_counter()
        ob.sptc(xs, self.X, [2, 3], [2, 3], max_products=10**10)
        return time.perf_counter() - t0

    def step(self) -> float:
        """Seconds of one baseline contraction of the sample."""
        if self.kind == "reference":
            t = run_sparta(self.xs_path, self.y_path, self.threads)
            if t is not None:
                return t
            self.kind, self.threads = "port", 1
        return self._port_time(self.xs)

    def describe(self, value: float) -> dict:
        return {"value": value, "unit": UNIT, "cores": self.threads, "kind": self.kind,
                "sample": f"{self.xs.nnz} X nonzeros (whole output rows, random) x full Y "
                          f"({self.X.nnz} nnz): {self.ir:.3e} matched products per run; "
                          + ("baselines/Sparta ttt EXPERIMENT_MODES=3, its [Total time]"
                             if self.kind == "reference" else "CPU oracle (ESC, FP64), wall time")}


def pct(v, p):
    """Nearest-rank percentile of sorted values."""
    return float(v[max(1, int(math.ceil(p / 100.0 * len(v)))) - 1])


def batched_stream(args, device, sp, stream):
    """The batched workload (256 independent contractions: orders 3-4, modes
    log-uniform 64..100k, nnz log-uniform 1e3..1e6, 1-2 contract modes, Zipf
    s in [1.0,1.4], U[-1,1), seed 3) run two ways on the same resident
    operands: plain (one gsparc_sptc per contraction, in order) and batched
    (one gsparc_sptc_batch)."""
    import torch
    import gsparc_b200 as gb
    from gsparc_b200 import synth
    inst = synth.batched_instances(args.mixed_count, seed=3, max_nnz=1_000_000)
    ctx = gb.Context(device)
    ctx.reserve()  # the pool mapped once, as for the headline contraction
    ops = [(ctx.upload(X, stream=sp), ctx.upload(Y, stream=sp)) for X, Y, _, _ in inst]
    jobs = [(dx, dy, cx, cy) for (dx, dy), (_, _, cx, cy) in zip(ops, inst)]
    nnz = sum(X.nnz + Y.nnz for X, Y, _, _ in inst)

    def plain_once(js=None):
        return sum(gb.sptc(ctx, dx, dy, cx, cy, 0, sink="discard", stream=sp).ir_nnz
                   for dx, dy, cx, cy in (jobs if js is None else js))

    def batched_once():
        res, bst = gb.sptc_batch(ctx, jobs, sink="discard", stream=sp)
        return bst

    # warm-up of both forms
    plain_once()
    batched_once()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    ir = plain_once()
    e1.record(stream)
    torch.cuda.synchronize()
    plain_ms = e0.elapsed_time(e1)
    e0.record(stream)
    bst = batched_once()
    e1.record(stream)
    torch.cuda.synchronize()
    batched_ms = e0.elapsed_time(e1)
    assert bst["ir_nnz"] == ir

    # the bound batching can reach: the ten largest instances (by matched
    # products) run plain, alone; batching cannot make the others cost less
    # than nothing, so plain_ms / top10_ms bounds batched_over_plain
    prods = [gb.sptc(ctx, dx, dy, cx, cy, 0, sink="discard", stream=sp).ir_nnz for dx, dy, cx, cy in jobs]
    top = sorted(range(len(jobs)), key=lambda i: -prods[i])[:10]
    e0.record(stream)
    plain_once([jobs[i] for i in top])
    e1.record(stream)
    torch.cuda.synchronize()
    top10_ms = e0.elapsed_time(e1)

    # planned and replayed: the coordinate-only work once (gsparc_plan_create),
    # then value refresh + every chunk's numeric pass captured in one CUDA graph
    # (the chunks share one output buffer, dropped like the discard sink's)
    t0 = time.perf_counter()
    plan = gb.Plan(ctx, jobs, max_chunk_nnz=1 << 30, stream=sp)
    plan_s = time.perf_counter() - t0
    cmax = max([plan.chunk(k)[1] for k in range(plan.nchunks)] + [1])
    okeys = torch.empty(cmax, dtype=torch.int64, device=stream.device)
    ovals = torch.empty(cmax, dtype=torch.float32, device=stream.device)
    gs_ = torch.cuda.Stream(device=stream.device)
    graph = torch.cuda.CUDAGraph()
    with torch.cuda.graph(graph, stream=gs_, capture_error_mode="relaxed"):
        plan.refresh(stream=gs_.cuda_stream)
        for k in range(plan.nchunks):
            plan.execute(k, okeys, ovals, stream=gs_.cuda_stream)
    graph.replay()  # warm-up
    torch.cuda.synchronize()
    g0, g1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(gs_):
        g0.record(gs_)
        graph.replay()
        g1.record(gs_)
    torch.cuda.synchronize()
    plan.check()
    replay_ms = g0.elapsed_time(g1)
    nchunks = plan.nchunks
    del graph
    plan.close()
    for dx, dy in ops:
        dx.free()
        dy.free()
    ctx.close()
    desc = (f"{len(jobs)} independent contractions, {nnz} operand nonzeros, {ir:.4e} matched products "
            "(orders 3-4, modes log-uniform 64..100k, nnz log-uniform 1e3..1e6, 1-2 contract modes, "
            "Zipf s 1.0-1.4, U[-1,1), seed 3)")
    return {"workload": desc, "unit": UNIT,
            "plain_value": ir / (plain_ms / 1e3), "plain_ms": plain_ms,
            "batched_value": ir / (batched_ms / 1e3), "batched_ms": batched_ms,
            "batched_over_plain": plain_ms / batched_ms, "groups_launches": bst["kernel_launches"],
            "top10_plain_ms": top10_ms, "top10_share_of_products": sum(prods[i] for i in top) / ir,
            "bound_over_plain": plain_ms / top10_ms,
            "replay_numeric_only_value": ir / (replay_ms / 1e3), "replay_numeric_only_ms": replay_ms,
            "replay_numeric_only_over_plain": plain_ms / replay_ms, "plan_create_ms": plan_s * 1e3,
            "replay": f"gsparc_plan: coordinate work once (plan_create_ms, host clock, not in replay_ms), then "
                      f"value refresh and the numeric pass of {nchunks} output chunks replayed from one CUDA graph: "
                      "numeric only, not comparable with plain_ms",
            "timing": "CUDA events on the launching stream, each form after one warm-up pass"}


def served_stream(args, device, sp, stream):
    """The served workload, bounded so a run stays within minutes: 256 requests
    with operand orders 3-5, 1-2 contract modes, modes log-uniform 64..100k,
    operand nnz from a power law n^-1.5 on [1e4, --served-max-nnz (2e6)], Zipf s in [1.0,1.4]
    indices, U[-1,1) values, Poisson arrivals at a mean 2000/s (seed 5), into
    a gsparc_serve_* server with a 150 GB budget (less if the GPU has less
    free); the plain form answers the same arrivals one at a time."""
    import torch
    import gsparc_b200 as gb
    from gsparc_b200 import synth
    inst, arrive = synth.served_stream(args.mixed_count, seed=5, max_nnz=int(args.served_max_nnz))
    nnz = sum(X.nnz + Y.nnz for X, Y, _, _ in inst)
    free_b, _ = torch.cuda.mem_get_info()
    budget = min(150 << 30, int(free_b * 0.8))

    def served_run(lanes):
        srv = gb.Server(device, hbm_budget=budget, lanes=lanes)
        sops = [(srv.upload(X), srv.upload(Y)) for X, Y, _, _ in inst]
        tickets = [None] * len(inst)

        def client():
            t0 = time.perf_counter()
            for i, ((sx, sy), (_, _, cx, cy)) in enumerate(zip(sops, inst)):
                d = t0 + arrive[i] - time.perf_counter()
                if d > 0:
                    time.sleep(d)
                tickets[i] = srv.submit(sx, sy, cx, cy, sink="discard")
        # one untimed pass of the same paced stream (the plain form gets a
        # warm-up pass too; both map their memory pools before it), then the
        # timed one
        for rep in range(2):
            srv.reset_stats()
            th = threading.Thread(target=client)
            th.start()
            th.join()
            for t in tickets:
                srv.wait(t)
        st = srv.stats()
        srv.close()
        return st
    sst = served_run(2)  # the server's default: two lanes
    sst1 = served_run(1)

    # plain form on the same arrivals: one contraction at a time, in order
    ctx = gb.Context(device, hbm_budget=budget)
    ctx.reserve()
    ops = [(ctx.upload(X, stream=sp), ctx.upload(Y, stream=sp)) for X, Y, _, _ in inst]
    jobs = [(dx, dy, cx, cy) for (dx, dy), (_, _, cx, cy) in zip(ops, inst)]
    ir = sum(gb.sptc(ctx, dx, dy, cx, cy, 0, sink="discard", stream=sp).ir_nnz for dx, dy, cx, cy in jobs)
    torch.cuda.synchronize()
    lat = []
    t0 = time.perf_counter()
    for i, (dx, dy, cx, cy) in enumerate(jobs):
        d = t0 + arrive[i] - time.perf_counter()
        if d > 0:
            time.sleep(d)
        gb.sptc(ctx, dx, dy, cx, cy, 0, sink="discard", stream=sp)
        lat.append((time.perf_counter() - t0 - arrive[i]) * 1e3)
    plain_wall = time.perf_counter() - t0
    lat = np.sort(np.asarray(lat))
    for dx, dy in ops:
        dx.free()
        dy.free()
    ctx.close()
    assert sst["ir_nnz"] == ir
    wide = sum(1 for X, Y, _, _ in inst
               if sum(synth._bits(d) for d in X.dims) > 64 or sum(synth._bits(d) for d in Y.dims) > 64)
    desc = (f"{len(inst)} requests, {nnz} operand nonzeros, {ir:.4e} matched products (operand orders 3-5, "
            f"1-2 contract modes, modes log-uniform 64..100k, nnz power law n^-1.5 on [1e4, {args.served_max_nnz:.0e}], "
            "Zipf s 1.0-1.4, "
            f"U[-1,1), {wide} with operand keys over 64 bits, seed 5); Poisson arrivals, mean 2000/s; "
            f"HBM budget {budget / 2**30:.0f} GiB")
    return {"workload": desc, "unit": UNIT, "value": sst["products_per_s"], "p50_ms": sst["p50_ms"],
            "p99_ms": sst["p99_ms"], "mean_ms": sst["mean_ms"], "wall_ms": sst["wall_ms"],
            "batches": sst["batches"], "max_batch": sst["max_batch"], "max_in_flight": sst["max_in_flight"],
            "plain_value": ir / plain_wall, "plain_p50_ms": pct(lat, 50), "plain_p99_ms": pct(lat, 99),
            "plain_wall_ms": plain_wall * 1e3, "served_over_plain": sst["products_per_s"] / (ir / plain_wall),
            "lanes": 2,
            "one_lane": {"value": sst1["products_per_s"], "p50_ms": sst1["p50_ms"], "p99_ms": sst1["p99_ms"],
                         "wall_ms": sst1["wall_ms"], "batches": sst1["batches"],
                         "served_over_plain": sst1["products_per_s"] / (ir / plain_wall)},
            "timing": "host clock: latency = submission to result delivered; the plain form runs "
                      "each request when it has arrived and the previous one finished"}


# --------------------------------------------------------------------------- arms
def dist_setup(args):
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        import torch
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
        pg = dist
    return world, rank, local, pg


REPORT_KEYS = ("Result NNZ", "SLITOM time", "Partition time", "SpTC(IdxMatch + Contraction + Data Copy) time",
               "Total time")


def run_report(binary, xp, yp, cx, cy, dense, iters=3, timeout=1200, extra=()):
    """Run a GSPARC-style CLI (-n iters); its stderr report as a dict (seconds per
    iteration, averaged by the program; the last section wins)."""
    cmd = [binary, "-X", xp, "-Y", yp, "-c", str(len(cx)), "-x", *map(str, cx), "-y", *map(str, cy),
           "-d", str(dense), "-n", str(iters), *extra]
    t0 = time.perf_counter()
    try:
        r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout)
    except subprocess.TimeoutExpired:
        return {"error": f"timed out after {timeout} s"}
    out = {"rc": r.returncode, "wall_s": round(time.perf_counter() - t0, 3)}
    for line in r.stderr.splitlines():
        for k in REPORT_KEYS:
            if line.startswith(k + ":"):
                out[k] = float(line.split(":", 1)[1])
    if r.returncode != 0:
        out["error"] = r.stderr[-400:]
    return out


def host_products(X, Y, cx, cy):
    """Matched products: per X nonzero, the number of Y nonzeros with its contract index."""
    def lin(T, modes):
        k = np.zeros(T.nnz, np.int64)
        for m in modes:
            k = k * int(T.dims[m]) + T.idx[m].astype(np.int64)
        return k
    xc, yc = lin(X, cx), lin(Y, cy)
    uc, cnt = np.unique(yc, return_counts=True)
    pos = np.minimum(np.searchsorted(uc, xc), len(uc) - 1)
    return int(np.where(uc[pos] == xc, cnt[pos], 0).sum())


def reference_gpu(args):
    """The reference GSPARC program (oracle/_ref/gsparc: its main.cu and src/ compiled
    unmodified for sm_100a) and our CLI, each run once on the same .tns files in
    ESC mode (-d -1; ours also in its default mode), timed by their own reports.
    The reference copies every output partition to pinned host memory
    (include/gsparc/contraction.cuh:554-555); ours does the same with -H (every
    output chunk to a page-locked host ring), which is the like-for-like
    comparison; ours without -H drops the output in HBM."""
    synth = synth_module()
    cli = os.path.join(ROOT, "gsparc_b200", "bin", "gsparc")
    ref = os.path.join(ROOT, "oracle", "_ref", "gsparc")
    if not os.path.exists(ref):
        print(json.dumps({"impl": "reference", "reference_gpu": {"unavailable": "oracle/_ref/gsparc not built"}}))
        return
    cases = [("plain_small", synth.plain_small), ("esc_large", synth.esc_large), ("dense_acc", synth.dense_acc)]
    res = {}
    clk = Clocks(0)
    clk.start()
    for name, make in cases:
        X, Y, cx, cy = make(scale=args.scale)
        d = tempfile.mkdtemp(prefix="gsparc_refgpu_")
        xp = os.path.join(d, "x.tns")
        synth.write_tns(xp, X)
        yp = xp
        if Y is not X:
            yp = os.path.join(d, "y.tns")
            synth.write_tns(yp, Y)
        ir = host_products(X, Y, cx, cy)
        row = {"nnz_x": X.nnz, "nnz_y": Y.nnz, "products": ir,
               "reference_esc": run_report(ref, xp, yp, cx, cy, -1),
               "ours_esc_host_copy": run_report(cli, xp, yp, cx, cy, -1, extra=["-H"]),
               "ours_auto_host_copy": run_report(cli, xp, yp, cx, cy, 0, extra=["-H"]),
               "ours_esc_in_hbm": run_report(cli, xp, yp, cx, cy, -1),
               "ours_auto_in_hbm": run_report(cli, xp, yp, cx, cy, 0)}
        for k in ("reference_esc", "ours_esc_host_copy", "ours_auto_host_copy", "ours_esc_in_hbm",
                  "ours_auto_in_hbm"):
            t = row[k].get("SpTC(IdxMatch + Contraction + Data Copy) time")
            if t:
                row[k]["products_per_s_sptc"] = ir / t
        res[name] = row
        print(json.dumps({name: row}), file=sys.stderr, flush=True)
        shutil.rmtree(d, ignore_errors=True)
    line = {"impl": "reference", "reference_gpu": {
        "binary": "oracle/_ref/gsparc: the reference main.cu + src/, unmodified, nvcc -gencode sm_100a",
        "timing": "each program's own stderr report (seconds per iteration, -n 3 averaged by the program, "
                  "device memory pools set up before the first iteration in both); the reference copies every "
                  "output partition to pinned host memory, ours with -H copies every output chunk to a "
                  "page-locked host ring (like for like), ours *_in_hbm drops the output in HBM",
        "scale": args.scale, "workloads": res}, "clocks": clk.stop()}
    print(json.dumps(line), flush=True)


def reference_arm(args, world, rank):
    if rank != 0:
        return
    if args.reference_gpu:
        reference_gpu(args)
        return
    X, _, cx, cy = workload(0, args.scale)
    # a step is a bounded sample (about 2 s of the baseline's own time) so that
    # the default --steps/--warmup run ends within a few minutes
    base = CpuBaseline(X, target_seconds=min(args.cpu_seconds, 2.0))
    for _ in range(args.warmup):
        base.step()
    ts = [base.step() for _ in range(args.steps)]
    t = float(np.mean(ts))
    value = base.ir / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": f"{WORKLOAD} sample", "contract": "-c 2 -x 2 3 -y 2 3",
                   "nnz": X.nnz, "dims": X.dims, "seed": 1, "sample_products": base.ir},
        "cpu_baseline": base.describe(value),
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


def ours_arm(args, world, rank, local, dist):
    import torch
    import gsparc_b200 as gb

    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    if args.served_only:
        stream = torch.cuda.current_stream(dev)
        if rank == 0:
            print(json.dumps({"served": served_stream(args, local, stream.cuda_stream, stream)}), flush=True)
        return
    # one contraction; with N ranks each contracts its row shard (rows of about
    # equal matched-product mass, the reference's per-GPU partition loop)
    X, _, cx, cy = workload(0, args.scale)
    ctx = gb.Context(local)
    stream = torch.cuda.current_stream(dev)
    sp = stream.cuda_stream
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=dev)
    # the context's memory pool is mapped once, before anything is timed, as the
    # reference's CudaMemoryPool takes the device memory once per run
    # (src/gsparc/cuda_memory.cpp:17-28) and the drop-in CLI does at start-up
    ctx.reserve()

    dX = ctx.upload(X, stream=sp)

    def step():
        return gb.sptc(ctx, dX, dX, cx, cy, 0, sink="discard", shard=rank, nshards=world, stream=sp)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    flush.zero_()  # the first GPU work after the sampler starts absorbs its start-up stall
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    stats = []
    e0.record(stream)
    for _ in range(args.steps):
        flush.zero_()  # inputs are < L2: write 256 MB between steps
        stats.append(step().stats)
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    clk = clocks.stop()
    ms = e0.elapsed_time(e1)
    ir = stats[0]["ir_nnz"]
    if dist is not None:
        t = torch.tensor([ms], dtype=torch.float64, device=dev)
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
        ms = float(t.item())
        n = torch.tensor([ir * args.steps], dtype=torch.float64, device=dev)
        dist.all_reduce(n)
        total_products = float(n.item())
    else:
        total_products = float(ir * args.steps)
    value = total_products / (ms / 1e3)

    # roofline of the contraction (sort + match + accumulate, every kernel of a
    # step), from the engine's own CUDA events: the algorithmic bytes of an ESC
    # contraction over its time
    s0 = stats[-1]
    peaks = load_peaks()
    t_step = float(np.mean([s["t_total_ms"] for s in stats]))
    alg = alg_bytes_contraction(X.nnz, X.order, X.nnz, X.order, ir, s0["nnz"])
    achieved = alg / (t_step / 1e3) / 1e9
    traffic = (TRAFFIC_NUMERIC_PER_OUTPUT * s0["nnz"]
               + TRAFFIC_PER_KEPT_BITMAP_BYTE * s0["kept_bitmap_bytes"]
               + TRAFFIC_OTHER_PER_OPERAND_NNZ * (s0["nnz_x"] + s0["nnz_y"]))
    roofline = {"bound": "hbm", "kernel": "the contraction: linearise, sort, match, planning, symbolic and "
                "numeric accumulation of every output chunk",
                "achieved": achieved, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                "frac": achieved / peaks["hbm_gbs"], "peak_source": peaks["source"],
                "traffic": traffic,
                "traffic_scope": "DRAM bytes read + written by every kernel of one contraction, from ncu "
                                 "captures at scale 0.1 scaled per output (numeric kernels), per kept bitmap "
                                 "byte (written by the symbolic pass, read by the numeric) and per operand "
                                 "nonzero (the rest)",
                "alg_bytes": alg,
                "alg_formula": "sum over X, Y of nnz*(8*order+4) + 24*nnz, + 16*nnz_X + 8*nnz_Y + 24*products "
                               "+ 12*nnz_Z",
                "ms_per_contraction": t_step, "units": "one contraction per launch of the path"}
    # the bytes this engine moves (it never writes a product to HBM): the output
    # once, the X match arrays and the Y rank / value once, over the numeric kernels
    t_num = float(np.mean([s["t_numeric_kernel_ms"] for s in stats]))
    moved = 12.0 * s0["nnz"] + 16.0 * s0["nnz_x"] + 8.0 * s0["nnz_y"]
    bytes_moved = {"kernel": "k_rowwin<numeric> + k_light<numeric> + k_stream",
                   "achieved": moved / (t_num / 1e3) / 1e9, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                   "frac": moved / (t_num / 1e3) / 1e9 / peaks["hbm_gbs"], "bytes_per_step": moved,
                   "kernel_ms_per_step": t_num, "launches_per_step": s0["chunks"],
                   "products_per_s_in_kernel": s0["ir_nnz"] / (t_num / 1e3)}
    launches = int(sum(s["kernel_launches"] for s in stats))

    # accuracy: one more contraction (untimed) with the engine's FP64 verification
    # on the GPU over a seeded sample of output rows of about 2^27 products
    ctx.set_verify(1 << 27)
    vst = step().stats
    ctx.set_verify(0)
    accuracy = {"max_rel_err": vst["max_rel_err"], "max_abs_err": vst["max_abs_err"],
                "verified_nnz": vst["verified_nnz"], "verified_products": vst["verified_products"],
                "mismatch": vst["verify_mismatch"], "of_nnz": vst["nnz"], "of_products": vst["ir_nnz"],
                "against": "FP64 sums of the exact products, formed on the GPU (untimed run)",
                "sample": "seeded sample of whole output rows, about 2^27 products"}

    # end to end through the public API: pinned host COO in, every output chunk out
    e2e = None
    if not args.no_e2e:
        dX.free()
        pin_idx = torch.from_numpy(X.idx.view(np.int64)).pin_memory()
        pin_val = torch.from_numpy(X.val).pin_memory()
        ring = 1 << 26
        hk = torch.empty(ring, dtype=torch.int64).pin_memory()
        hv = torch.empty(ring, dtype=torch.float32).pin_memory()
        hk_np = hk.numpy().view(np.uint64)
        hv_np = hv.numpy()

        class _Host:
            pass
        host = _Host()
        host.dims, host.idx, host.val = X.dims, pin_idx, pin_val

        def e2e_step():
            t = gb.DeviceTensor(ctx, host, stream=sp)
            r = gb.sptc(ctx, t, t, cx, cy, 0, sink="ring", host_keys=hk_np, host_vals=hv_np, shard=rank,
                        nshards=world, stream=sp)
            t.free()
            return r
        e2e_step()
        torch.cuda.synchronize()
        barrier()
        ks = max(1, min(args.steps, 3))
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        f0.record(stream)
        rs = [e2e_step() for _ in range(ks)]
        f1.record(stream)
        torch.cuda.synchronize()
        barrier()
        ems = f0.elapsed_time(f1)
        if dist is not None:
            t = torch.tensor([ems], dtype=torch.float64, device=dev)
            dist.all_reduce(t, op=dist.ReduceOp.MAX)
            ems = float(t.item())
        e2e_value = (total_products / args.steps) * ks / (ems / 1e3)
        h2d = X.nnz * (8 * X.order + 4)
        d2h = int(rs[-1].stats["bytes_d2h"])
        e2e = {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": ems / ks, "steps": ks,
               "sink": f"pinned host ring of {ring} nonzeros, every output chunk copied"}

    ctx.close()  # returns the large workload's memory before the mixed stream
    batched = served = None
    if world == 1 and not args.no_mixed:
        batched = batched_stream(args, local, sp, stream)
        served = served_stream(args, local, sp, stream)

    cpu = None
    if world == 1 and not args.no_cpu_baseline:
        base = CpuBaseline(X, target_seconds=args.cpu_seconds)
        cpu = base.describe(base.ir / base.step())

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "contract": "-c 2 -x 2 3 -y 2 3", "dims": X.dims,
                       "nnz": X.nnz, "seed": 1, "scale": args.scale,
                       "matched_products_per_step": int(total_products / args.steps),
                       "output_nnz_per_step_rank0": s0["nnz"],
                       "output_chunks": s0["chunks"], "l2": "256 MB flush write between steps",
                       "memory_pool": "mapped once before the warm-up (gsparc_ctx_reserve), as the reference's "
                                      "pool is",
                       "kept_bitmap_bytes": s0["kept_bitmap_bytes"],
                       "accumulator": "auto (dense window for heavy rows, on-chip ESC for light)",
                       "parallelism": f"{world} row shard(s) of one contraction, one per GPU, balanced by "
                                      "matched products; operands replicated; no data-path collective"},
            "roofline": roofline,
            "roofline_bytes_moved": bytes_moved,
            "accuracy": accuracy,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": launches,
            "clocks": clk,
            "batched": batched,
            "served": served,
            "heavy_windows": s0["heavy_windows"], "heavy_rows": s0["heavy_rows"], "rows": s0["rows"],
            "stage_ms": {k: s0[k] for k in ("t_linearize_ms", "t_sort_ms", "t_match_ms", "t_plan_ms",
                                             "t_contract_ms", "t_total_ms")},
            "step_total_ms": [round(s["t_total_ms"], 3) for s in stats],
        }
        print(json.dumps(line), flush=True)


def main():
    args = parse()
    world, rank, local, dist = dist_setup(args)
    try:
        if args.impl == "reference":
            reference_arm(args, world, rank)
        else:
            ours_arm(args, world, rank, local, dist)
    finally:
        if dist is not None:
            dist.destroy_process_group()


if __name__ == "__main__":
    main()

#!/usr/bin/env python
"""Benchmark of Catmull-Clark halfedge refinement on B200.

Workload (one "step"): ``ccs_Refine_Scatter`` of the mixed-crease torus cage
(64x64 grid-torus with triangles, pentagons, a boundary strip, crease chains
and UVs; H0 = 17,416 halfedges) to depth 6: topology, creases, UVs and FP32
points of every level, 95.1M refined halfedges per step.

Metric: refined halfedges per second (sum of H_d over depths 1..6 per step).

* ``value``   device time of the refine call with its inputs resident in HBM,
              CUDA events on the subd's stream, L2 flushed (256 MB write)
              between timed steps, outside the events.
* ``e2e``     the same call through the C ABI with host buffers: upload of
              the cage points from pinned host memory, refine, download of
              every level's halfedges, creases and points to the host.
* ``roofline`` the kernel with the largest share of device time (per-launch
              CUDA events inside the library), its algorithmic bytes per
              launch over its mean duration, against MEASURED_PEAKS.json.
* ``cpu_baseline`` the reference's own ccs_Refine_Scatter (compiled from its
              sources into oracle/_ref, OpenMP on all host cores) on the same
              cage and depth, a bounded sample of runs.

``--op points`` times ccs_RefineVertexPoints_Scatter_cuda on the refined
topology instead (the call of an animation or fitting loop); its e2e moves
the cage points in and the points of every depth out through the
differentiable entry point, and its cpu_baseline is the reference's
ccs_RefineVertexPoints_Scatter.
``batch`` (default line): the batched workload -- 512 uneven cages, forward
points + loss gradient + adjoint, batched (one persistent launch per depth)
against a Python loop of the single-mesh calls on the same GPU -- measured
after the headline refine in the same run (``--no-batch`` leaves it off).
``--impl reference`` times only the reference CPU path (rank 0).
Multi-GPU (torchrun): every rank refines its own replica of the cage (the
single-mesh path does not shard); value = all ranks' halfedges / max time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
if ROOT not in sys.path:
    sys.path.insert(0, ROOT)

METRIC = "refined halfedges/s"
UNIT = "halfedges/s"
L2_FLUSH_BYTES = 256 << 20


def parse():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=20)
    p.add_argument("--warmup", type=int, default=5)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--depth", type=int, default=None,
                   help="refinement depth (default: 6 for mixed_torus, 5 for height_grid)")
    p.add_argument("--cpu-seconds", type=float, default=15.0)
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--e2e-steps", type=int, default=5)
    p.add_argument("--deterministic", action="store_true")
    p.add_argument("--op", default="refine", choices=["refine", "points"],
                   help="refine: ccs_Refine_Scatter_cuda (topology, creases, UVs, points); points: "
                        "ccs_RefineVertexPoints_Scatter_cuda on a refined topology (the call of an "
                        "animation or fitting loop)")
    p.add_argument("--workload", default="mixed_torus", choices=["mixed_torus", "height_grid", "batch"],
                   help="mixed_torus: the headline single-mesh refine (64x64 mixed-valence torus, "
                        "depth 6); height_grid: the large plain refine (256x256 height-field grid, "
                        "depth 5, per-level GB/s); batch: 512 uneven cages, forward + adjoint, "
                        "batched vs a loop of single-mesh calls")
    p.add_argument("--batch-count", type=int, default=512)
    p.add_argument("--no-batch", action="store_true",
                   help="leave the batched workload's measurement off the default line")
    return p.parse_args()


def workload(args):
    from halfedgecatmullclark_b200 import configs
    if args.workload == "height_grid":
        return configs.height_grid(depth=5 if args.depth is None else args.depth)
    return configs.mixed_torus(depth=6 if args.depth is None else args.depth)


WORKLOAD_NAMES = {"mixed_torus": "mixed_torus_64x64_depth%d", "height_grid": "height_grid_256x256_depth%d"}


def config_dict(w, extra=None):
    c = {"workload": WORKLOAD_NAMES.get(w.name, w.name + "_depth%d") % w.depth, "cage_halfedges": w.cage.H,
         "cage_faces": w.cage.F, "depth": w.depth, "uv": w.cage.U > 0,
         "crease_edges": w.notes.get("crease_edges"), "l2": "flushed (256 MB write) between timed steps"}
    if extra:
        c.update(extra)
    return c


# ---------------------------------------------------------------------------
# clocks sampled during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    """SM clock, power and clock-event reasons of this process's GPU, sampled
    while the timed region runs: NVML read every 2 ms on a thread (nothing is
    set), else `nvidia-smi -lms 200`."""
    QUERY = ("index,uuid,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    # NVML clock-event reason bits
    REASON_BITS = {"hw_slowdown": 0x8, "hw_thermal_slowdown": 0x40, "sw_thermal_slowdown": 0x20,
                   "sw_power_cap": 0x4}

    def __init__(self, uuid=None):
        self.uuid = uuid
        self.proc = None
        self.path = None
        self.thread = None
        self.rows = []

    def _nvml_handle(self):
        import pynvml
        pynvml.nvmlInit()
        if self.uuid:
            want = self.uuid.lower().replace("gpu-", "")
            for i in range(pynvml.nvmlDeviceGetCount()):
                h = pynvml.nvmlDeviceGetHandleByIndex(i)
                u = pynvml.nvmlDeviceGetUUID(h)
                u = (u.decode() if isinstance(u, bytes) else u).lower().replace("gpu-", "")
                if u == want:
                    return pynvml, h
        return pynvml, pynvml.nvmlDeviceGetHandleByIndex(0)

    def start(self):
        try:
            import threading
            nv, h = self._nvml_handle()
            self.smax = float(nv.nvmlDeviceGetMaxClockInfo(h, nv.NVML_CLOCK_SM))
            self.stop_flag = threading.Event()

            def run():
                while not self.stop_flag.is_set():
                    try:
                        self.rows.append((float(nv.nvmlDeviceGetClockInfo(h, nv.NVML_CLOCK_SM)),
                                          nv.nvmlDeviceGetPowerUsage(h) / 1000.0,
                                          int(nv.nvmlDeviceGetCurrentClocksEventReasons(h))))
                    except Exception:
                        break
                    time.sleep(0.002)
            self.thread = threading.Thread(target=run, daemon=True)
            self.thread.start()
            return
        except Exception:
            self.thread = None
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.fh = open(self.path, "w")
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.QUERY,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=self.fh, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def _stop_nvml(self):
        self.stop_flag.set()
        self.thread.join(timeout=5)
        try:
            import pynvml
            pynvml.nvmlShutdown()
        except Exception:
            pass
        rows = self.rows
        if not rows:
            return None
        pmax = max(r[1] for r in rows)
        load = [r[0] for r in rows if r[1] > 0.35 * pmax] or [r[0] for r in rows]
        reasons = sorted({n for r in rows for n, bit in self.REASON_BITS.items() if r[2] & bit})
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": self.smax, "reasons": reasons,
                "samples": len(rows), "power_w_max": pmax, "source": "nvml, 2 ms"}

    def stop(self):
        if self.thread is not None:
            return self._stop_nvml()
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.fh.close()
        rows = []
        with open(self.path) as fh:
            for line in fh:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) < 10:
                    continue
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        if self.uuid:
            mine = [r for r in rows if r[1].lower().endswith(self.uuid.lower()[-12:])]
            rows = mine or rows
        # keep the GPU that drew the most power (the one under load)
        by_idx = {}
        for r in rows:
            by_idx.setdefault(r[0], []).append(r)

        def pw(rs):
            try:
                return max(float(r[4]) for r in rs)
            except ValueError:
                return 0.0
        rs = max(by_idx.values(), key=pw)
        sm = [float(r[2]) for r in rs if r[2].replace(".", "").isdigit()]
        smax = [float(r[3]) for r in rs if r[3].replace(".", "").isdigit()]
        pmax = pw(rs)
        load = [s for s, r in zip(sm, rs) if float(r[4] or 0) > 0.35 * pmax] or sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rs for k in range(4) if "Active" in r[6 + k] and "Not" not in r[6 + k]})
        return {"sm_mhz": statistics.median(load) if load else None,
                "sm_max_mhz": max(smax) if smax else None, "reasons": reasons,
                "samples": len(rs), "power_w_max": pmax, "source": "nvidia-smi, 200 ms"}


def measured_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def traffic_table():
    """dram bytes per launch from the committed ncu summary, if present."""
    path = os.path.join(ROOT, "profiles", "traffic.json")
    try:
        with open(path) as fh:
            return json.load(fh)
    except Exception:
        return {}


# ---------------------------------------------------------------------------
# CPU baseline: the reference compiled from its sources (oracle/_ref)
# ---------------------------------------------------------------------------
def cpu_reference(w, seconds, max_runs=20, min_runs=2, op="refine"):
    from oracle import refimpl
    from halfedgecatmullclark_b200 import metrics
    from halfedgecatmullclark_b200.subd import level_counts
    sh = metrics.total_halfedges(level_counts(w.cage, w.depth))
    cores = os.cpu_count() or 1
    if refimpl.available():
        refimpl.set_threads(cores)
        s = refimpl.RefSubd(w.cage, w.depth)
        times = []
        passes = {}
        try:
            if op == "points":
                s.refine("scatter")                     # the topology, untimed
            t_end = time.perf_counter() + seconds
            while len(times) < max_runs and (len(times) < min_runs or time.perf_counter() < t_end):
                t0 = time.perf_counter()
                if op == "points":
                    s.call("ccs_RefineVertexPoints_Scatter")
                else:
                    s.refine("scatter")
                times.append(time.perf_counter() - t0)
            # its four passes one by one, as the reference's bench_cpu times them
            # (examples/subd_cpu.c:220-261); three runs each, median
            for name, fn in (("halfedges", "ccs_RefineHalfedges"), ("creases", "ccs_RefineCreases"),
                             ("vertex_uvs", "ccs_RefineVertexUvs"),
                             ("vertex_points", "ccs_RefineVertexPoints_Scatter")):
                pt = []
                for _ in range(3):
                    t0 = time.perf_counter()
                    s.call(fn)
                    pt.append(time.perf_counter() - t0)
                passes[name] = statistics.median(pt) * 1e3
        finally:
            s.close()
        med = statistics.median(times)
        return {"value": sh / med, "unit": UNIT, "cores": cores, "kind": "reference",
                "sample": "%d runs of the reference %s on the full workload "
                          "(OpenMP %d threads), median %.1f ms"
                          % (len(times), "ccs_RefineVertexPoints_Scatter" if op == "points" else "ccs_Refine_Scatter",
                             cores, med * 1e3),
                "ms_per_step": med * 1e3, "passes_ms": passes}
    # the oracle port, single-threaded, on a smaller depth of the same cage
    from oracle import oracle
    d = max(1, w.depth - 2)
    sh_d = metrics.total_halfedges(level_counts(w.cage, d))
    times = []
    t_end = time.perf_counter() + seconds
    while len(times) < max_runs and (len(times) < min_runs or time.perf_counter() < t_end):
        t0 = time.perf_counter()
        oracle.refine(w.cage, d, "scatter")
        times.append(time.perf_counter() - t0)
    med = statistics.median(times)
    return {"value": sh_d / med, "unit": UNIT, "cores": 1, "kind": "port",
            "sample": "%d runs of the single-threaded oracle at depth %d of the same cage" % (len(times), d),
            "ms_per_step": med * 1e3}


def run_reference(args):
    """The reference's own ccs_Refine_Scatter (or its points pass) on the same
    workload, OpenMP on every host core.  Nothing of the CUDA package's
    native code loads in this process: the cage comes from the reference's
    LoadObj on the workload's OBJ text (the same cage, byte for byte, as the
    CUDA arm's converter gives), and the halfedge total from the reference's
    own ccs_CumulativeHalfedgeCountAtDepth."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    if args.workload == "batch":
        print(json.dumps({"impl": "reference", "unavailable":
                          "the reference has neither an adjoint nor a batched path, so the batched "
                          "forward + adjoint cages/s has no reference run; the CUDA arm's line carries "
                          "its baseline (a loop of single-mesh calls on the same GPU)"}))
        return 0
    w = workload(args)
    from oracle import refimpl
    cores = os.cpu_count() or 1
    if not refimpl.available():
        from halfedgecatmullclark_b200 import metrics
        from halfedgecatmullclark_b200.subd import level_counts
        sh = metrics.total_halfedges(level_counts(w.cage, w.depth))
        cfg = config_dict(w, {"parallelism": "replicas x%d" % max(1, args.gpus),
                              "deterministic": bool(args.deterministic), "op": args.op,
                              "refined_halfedges_per_step": sh})
        base = cpu_reference(w, args.cpu_seconds, op=args.op)
        line = {"impl": "reference", "metric": METRIC, "value": base["value"], "unit": UNIT,
                "n_gpus": args.gpus, "steps": 0, "warmup": 0, "ms_per_step": base["ms_per_step"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": cfg, "cpu_baseline": base,
                "e2e": {"value": base["value"], "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
        print(json.dumps(line))
        return 0
    refimpl.set_threads(cores)
    cage = refimpl.cage_from_obj_text(w.obj())
    s = refimpl.RefSubd(cage, w.depth)
    sh = int(s.cumH)                               # halfedges of depths 1..D
    # the same config object as the CUDA arm's own line
    cfg = config_dict(w, {"parallelism": "replicas x%d" % max(1, args.gpus),
                          "deterministic": bool(args.deterministic), "op": args.op,
                          "refined_halfedges_per_step": sh})
    call = "ccs_RefineVertexPoints_Scatter" if args.op == "points" else "ccs_Refine_Scatter"
    try:
        if args.op == "points":
            s.refine("scatter")                     # the topology, untimed
        for _ in range(args.warmup):
            s.call(call)
        times = []
        for _ in range(args.steps):
            t0 = time.perf_counter()
            s.call(call)
            times.append(time.perf_counter() - t0)
    finally:
        s.close()
    total = sum(times)
    value = sh * args.steps / total
    line = {"impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": total / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": cfg,
            "cpu_baseline": {"value": value, "unit": UNIT, "cores": cores, "kind": "reference",
                             "sample": "%d timed runs of the reference %s on the full "
                                       "workload (cage by the reference's LoadObj), OpenMP %d threads"
                                       % (args.steps, call, cores)},
            "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line))
    return 0


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def dist_init():
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300),
                                device_id=torch.device("cuda", local))
    return rank, world


def barrier(world):
    if world > 1:
        import torch.distributed as dist
        dist.barrier()


def max_over_ranks(x, world):
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([x], dtype=torch.float64, device="cuda")
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def adjoint_timing(subd, w, stream, flush, steps, torch, peak=None):
    """Device ms of one adjoint pass (ccs_AdjointPointsDevice_cuda) and its
    per-kernel profile, on the workload's subd (topology already refined);
    the one-pass steps at depth >= 2 carry their algorithmic bytes
    (metrics.kernel_bytes("adj_step")) and fraction of `peak` GB/s."""
    import ctypes
    g = torch.randn((subd.cumV, 3), device="cuda")
    gc = torch.empty((w.cage.V, 3), device="cuda")
    sp = ctypes.c_void_p(int(stream.cuda_stream))
    call = lambda: subd.L.ccs_AdjointPointsDevice_cuda(subd.ptr, g.data_ptr(), gc.data_ptr(), sp)
    with torch.cuda.stream(stream):
        for _ in range(3):
            call()
    torch.cuda.synchronize()
    ms = []
    with torch.cuda.stream(stream):
        for _ in range(max(1, steps)):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            call()
            b.record(stream)
            ms.append((a, b))
    torch.cuda.synchronize()
    mean = statistics.mean(a.elapsed_time(b) for a, b in ms)
    subd.set_profiling(True)
    with torch.cuda.stream(stream):
        flush.zero_()
        call()
    recs = subd.read_profile(1 << 14)
    subd.set_profiling(False)
    by = {}
    for r in recs:
        by[(r["kernel"], r["level"])] = by.get((r["kernel"], r["level"]), 0.0) + r["ms"]
    top = sorted(by.items(), key=lambda kv: -kv[1])[:10]
    from halfedgecatmullclark_b200 import metrics
    kernels = []
    for (name, level), v in top:
        e = {"kernel": name, "level": level, "ms": v}
        if name == "adj_step" and peak:
            nb = metrics.kernel_bytes("adj_step", subd.levels[level], 4 * subd.record_words)
            e.update({"alg_bytes": nb, "gbs": nb / (v / 1e3) / 1e9, "frac_of_peak": nb / (v / 1e3) / 1e9 / peak})
        kernels.append(e)
    return {"ms_per_pass": mean, "halfedges_per_s": subd_halfedges(subd) / (mean / 1e3), "kernels": kernels}


def subd_halfedges(subd):
    from halfedgecatmullclark_b200 import metrics
    return metrics.total_halfedges(subd.levels)


def batch_measure(args, rank, world):
    """Many uneven cages (512 by default: faces log-uniform in [50, 5000],
    depths uniform in {2..6}); one step = forward (points), the gradient of
    the fitting loss (mean squared distance to a fixed target), adjoint.
    Batched (one persistent launch per depth, CUDA graph, autotuned grid)
    against a Python loop of the single-mesh C-ABI calls on the same GPU and
    stream; both arms compute the loss gradient as one elementwise operation.
    Under torchrun every rank refines its own shard of the cages (no
    exchange); times are the max over ranks.  Returns the measurement on
    rank 0 (None elsewhere)."""
    import ctypes
    import torch
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200 import batch as B
    from halfedgecatmullclark_b200 import configs
    from halfedgecatmullclark_b200 import shard
    from halfedgecatmullclark_b200.subd import Subd

    ws_all = configs.batch_cages(count=args.batch_count)
    # independent cages: each rank refines its own share, no exchange
    parts = shard.shard([shard.cage_work(w.cage, w.depth) for w in ws_all], world)
    ws = [ws_all[i] for i in parts[rank]]
    cages = [w.cage for w in ws]
    depths = [w.depth for w in ws]
    stream = torch.cuda.Stream()
    sp = ctypes.c_void_p(int(stream.cuda_stream))
    steps = max(1, args.steps)

    # loop of single-mesh calls (pageable host arrays: nothing is downloaded)
    subds = []
    for w in ws:
        s = Subd(w.cage, w.depth, N.FLAG_PAGEABLE_HOST)
        s.set_stream(stream)
        s.refine_halfedges()
        s.refine_creases()
        subds.append(s)
    # the points and gradients of every cage in one buffer each, cages one
    # after the other (the batch's own layout), so that the loss gradient is
    # one elementwise operation in both arms
    total = sum(s.cumV for s in subds)
    P_all = torch.empty((total, 3), device="cuda")
    G_all = torch.empty((total, 3), device="cuda")
    GC_all = torch.empty((sum(s.cage.V for s in subds), 3), device="cuda")
    bufs = []
    off = offc = 0
    for s in subds:
        x = torch.tensor(s.cage.vertex_points, device="cuda")
        gc = GC_all[offc:offc + s.cage.V]
        bufs.append((x, P_all[off:off + s.cumV], G_all[off:off + s.cumV], gc))
        off += s.cumV
        offc += s.cage.V
    L = N.lib()
    # the fitting loss: mean squared distance of the refined points to a
    # fixed seeded target of unit scale (independent of P, so that P - T
    # carries no cancellation and the two arms' gradients stay comparable);
    # its gradient 2 (P - T) / N reaches the cage through the adjoint, which
    # is linear: both arms feed it P - T (one elementwise pass over every
    # point) and scale the cage points' gradient by 2 / N afterwards
    scale = 2.0 / total
    T_all = torch.randn((total, 3), device="cuda", generator=torch.Generator("cuda").manual_seed(5))

    def loss_grad(P, G):
        torch.sub(P, T_all, out=G)

    def loop_step():
        for s, (x, p, g, gc) in zip(subds, bufs):
            L.ccs_RefinePointsDevice_cuda(s.ptr, x.data_ptr(), p.data_ptr(), 0, sp)
        with torch.cuda.stream(stream):
            loss_grad(P_all, G_all)
        for s, (x, p, g, gc) in zip(subds, bufs):
            L.ccs_AdjointPointsDevice_cuda(s.ptr, g.data_ptr(), gc.data_ptr(), sp)
        with torch.cuda.stream(stream):
            GC_all.mul_(scale)

    torch.cuda.synchronize()
    for _ in range(max(3, args.warmup)):
        loop_step()
    torch.cuda.synchronize()
    barrier(world)
    a = torch.cuda.Event(enable_timing=True)
    b = torch.cuda.Event(enable_timing=True)
    a.record(stream)
    for _ in range(steps):
        loop_step()
    b.record(stream)
    torch.cuda.synchronize()
    loop_ms = shard.max_over_ranks(a.elapsed_time(b) / steps, world)
    loop_sample = [bufs[i][3].clone() for i in (0, len(bufs) // 2, len(bufs) - 1)]
    # the same loop captured into one CUDA graph and replayed: its launches
    # no longer pay the host's per-call cost, so the ratio loop_ms /
    # graph_ms bounds what removing that cost alone (batching or not) can win
    graph_ms = None
    try:
        g = torch.cuda.CUDAGraph()
        with torch.cuda.graph(g, stream=stream):
            loop_step()
        for _ in range(2):
            g.replay()
        torch.cuda.synchronize()
        a.record(stream)
        with torch.cuda.stream(stream):
            for _ in range(steps):
                g.replay()
        b.record(stream)
        torch.cuda.synchronize()
        graph_ms = shard.max_over_ranks(a.elapsed_time(b) / steps, world)
        del g
    except Exception as exc:  # the captured loop is a reference figure only
        graph_ms = None
        print("loop capture failed: %s" % exc, file=sys.stderr)
    for s in subds:
        s.close()
    del bufs, P_all, G_all, GC_all
    subds.clear()
    torch.cuda.empty_cache()

    bt = B.Batch(cages, depths)
    bt.set_stream(stream)
    ta = torch.cuda.Event(enable_timing=True)
    tb = torch.cuda.Event(enable_timing=True)
    ta.record(stream)
    bt.refine()
    tb.record(stream)
    bt.synchronize()
    topo_ms = ta.elapsed_time(tb)
    tune = B.autotune(bt, use_cache=False, iters=2, stream=stream)
    bt.set_stream(stream)
    arr = bt.arrays()
    assert T_all.shape == arr["points"].shape      # the batch stores cages one after the other

    def batch_step():
        bt.refine_points()
        # the adjoint of P - T with the finest levels' P - T formed inside its
        # first step (ccs_BatchAdjointDistance_cuda); the loop forms P - T in
        # one elementwise pass and feeds it to the plain adjoint
        bt.adjoint_distance(T_all)
        arr["grad_cage_points"].mul_(scale)

    with torch.cuda.stream(stream):
        for _ in range(max(3, args.warmup)):
            batch_step()
    bt.synchronize()
    barrier(world)
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(torch.cuda.current_device()).uuid)
    except Exception:
        pass
    sampler = ClockSampler(uuid)
    sampler.start()
    with torch.cuda.stream(stream):
        a.record(stream)
        for _ in range(steps):
            batch_step()
        b.record(stream)
    bt.synchronize()
    clocks = sampler.stop()
    batch_ms = shard.max_over_ranks(a.elapsed_time(b) / steps, world)
    # gradients of the last full step (the adjoint consumes its input, so
    # before the halves are timed alone)
    agree = max(float((arr["grad_cage_points"][bt.cage_slice(i)] - ref).abs().max() /
                      max(ref.abs().max(), 1e-30))
                for i, ref in zip((0, len(ws) // 2, len(ws) - 1), loop_sample))
    # the parts alone (same stream, CUDA events)
    parts = {}
    for name, fn in (("forward_ms", bt.refine_points), ("adjoint_ms", lambda: bt.adjoint_distance(T_all)),
                     ("loss_grad_ms", lambda: loss_grad(arr["points"], arr["grad_points"]))):
        with torch.cuda.stream(stream):
            a.record(stream)
            for _ in range(steps):
                fn()
            b.record(stream)
        bt.synchronize()
        parts[name] = shard.max_over_ranks(a.elapsed_time(b) / steps, world)
    agree = shard.max_over_ranks(agree, world)
    sh = int(shard.sum_over_ranks(sum(inf["halfedgeCount"] for inf in bt.info), world))
    topo_ms = shard.max_over_ranks(topo_ms, world)
    bt.close()
    del arr
    torch.cuda.empty_cache()
    if rank != 0:
        return None
    return {"metric": "batched forward+adjoint cages/s", "value": len(ws_all) / (batch_ms / 1e3),
            "unit": "cages/s", "ms_per_step": batch_ms, "steps": steps,
            "config": {"workload": "batch_cages_%d" % len(ws_all), "faces": "log-uniform [50, 5000]",
                       "depths": "uniform {2..6}", "refined_halfedges": sh,
                       "parallelism": "cage shards x%d (no exchange)" % world,
                       "schedule": {"blocks_per_sm": tune["blocks_per_sm"], "split": tune.get("split"),
                                    "tried": tune["tried"]}},
            "loop": {"value": len(ws_all) / (loop_ms / 1e3), "unit": "cages/s", "ms_per_step": loop_ms,
                     "graph_ms": graph_ms,
                     "max_speedup_from_launch_cost": loop_ms / graph_ms if graph_ms else None,
                     "how": "Python loop of ccs_RefinePointsDevice_cuda per cage, the loss gradient over "
                            "all cages' points in one op, then ccs_AdjointPointsDevice_cuda per cage; "
                            "graph_ms = the same calls captured in one CUDA graph and replayed (no "
                            "host cost per call)"},
            "speedup_vs_loop_graph": graph_ms / batch_ms if graph_ms else None,
            "speedup_vs_loop": loop_ms / batch_ms, "topology_refine_ms": topo_ms,
            "forward_ms": parts["forward_ms"], "adjoint_ms": parts["adjoint_ms"],
            "loss_grad_ms": parts["loss_grad_ms"],
            "grad_agreement_rel": agree, "clocks": clocks,
            "step": "forward points, gradient of the mean squared distance to a fixed target, adjoint; "
                    "the adjoint is linear, so both arms feed it P - T and scale the cage gradient by 2/N. "
                    "Loop: P - T in one elementwise pass, then the per-cage adjoints. Batch: "
                    "ccs_BatchAdjointDistance_cuda, the finest levels' P - T formed inside the first "
                    "adjoint step (adjoint_ms includes its elementwise part; loss_grad_ms is the loop's pass)"}


def run_batch_workload(args):
    """The batched workload as the line's own metric (--workload batch)."""
    rank, world = dist_init()
    m = batch_measure(args, rank, world)
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    if rank != 0:
        return 0
    line = {"metric": m["metric"], "value": m["value"], "unit": m["unit"], "n_gpus": world,
            "steps": m["steps"], "warmup": args.warmup, "ms_per_step": m["ms_per_step"],
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": m["config"]}
    line.update({k: v for k, v in m.items() if k not in line and k != "metric"})
    print(json.dumps(line))
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload == "batch":
        return run_batch_workload(args)
    import torch
    from halfedgecatmullclark_b200 import _native as N
    from halfedgecatmullclark_b200 import metrics
    from halfedgecatmullclark_b200.subd import Subd

    rank, world = dist_init()
    w = workload(args)
    flags = N.FLAG_DETERMINISTIC if args.deterministic else 0
    subd = Subd(w.cage, w.depth, flags)
    stream = torch.cuda.Stream()
    subd.set_stream(stream)
    points_op = args.op == "points"
    if points_op:
        def step():
            subd.refine_vertex_points("scatter")
    else:
        step = subd.refine_scatter
    levels = subd.levels
    SH = metrics.total_halfedges(levels)
    flush = torch.empty(L2_FLUSH_BYTES, dtype=torch.uint8, device="cuda")
    uuid = None
    try:
        uuid = str(torch.cuda.get_device_properties(torch.cuda.current_device()).uuid)
    except Exception:
        pass

    with torch.cuda.stream(stream):
        if points_op:
            subd.refine_scatter()              # the topology the points step needs, untimed
        for _ in range(max(3, args.warmup)):
            step()
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()

    sampler = ClockSampler(uuid)
    sampler.start()
    t_wall = time.perf_counter()
    evs = []
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()
            a = torch.cuda.Event(enable_timing=True)
            b = torch.cuda.Event(enable_timing=True)
            a.record(stream)
            step()
            b.record(stream)
            evs.append((a, b))
    torch.cuda.synchronize()
    barrier(world)
    torch.cuda.synchronize()
    wall = time.perf_counter() - t_wall
    clocks = sampler.stop()
    step_ms = [a.elapsed_time(b) for a, b in evs]
    total_ms = max_over_ranks(sum(step_ms), world)

    # per-kernel device times: the same refine replayed as a profiled CUDA
    # graph whose event record nodes time every launch as the graph runs it
    subd.set_profiling(True)
    with torch.cuda.stream(stream):
        for _ in range(args.steps):
            flush.zero_()
            step()
    recs = subd.read_profile(1 << 16)
    subd.set_profiling(False)

    value = world * SH * args.steps / (total_ms / 1e3)
    rec_bytes = 16 if subd.record_words == 4 else 12

    # roofline of the dominant kernel
    by = {}
    units = {}
    for r in recs:
        by.setdefault((r["kernel"], r["level"]), []).append(r["ms"])
        units[(r["kernel"], r["level"])] = r["units"]
    steps_by = {k: v for k, v in by.items() if k[0] == "step"}
    by = {k: v for k, v in by.items() if k[0] != "step"}
    total_prof = sum(sum(v) for v in by.values())
    # the dominant kernel of the subd's own stream (ring_stats runs on the
    # second stream beside kernel A: its events span the overlap)
    dom_key = max((k for k in by if k[0] not in ("ring_stats", "crease_stats", "cage_side")),
                  key=lambda k: sum(by[k]))
    dom_ms = statistics.mean(by[dom_key])
    def kbytes(kernel, d):
        u = units.get((kernel, d)) if kernel in ("cage_side", "ring_stats") and d == 0 else None
        if kernel in ("exact_points", "old_vertices"):
            u = units.get(("old_vertices", d))
        return metrics.kernel_bytes(kernel, levels[d], rec_bytes, levels[d - 1] if d >= 1 else None, u)
    dom_bytes = kbytes(*dom_key)
    peak, peak_kind = measured_peak()
    achieved = dom_bytes / (dom_ms / 1e3) / 1e9
    traffic = traffic_table().get("%s@%d" % dom_key)
    kernels = sorted(({"kernel": k[0], "level": k[1], "mean_ms": statistics.mean(v),
                       "share": sum(v) / total_prof,
                       "gbs": kbytes(*k) / (statistics.mean(v) / 1e3) / 1e9}
                      for k, v in by.items()), key=lambda x: -x["share"])
    per_depth = []
    for d in range(w.depth):
        # a whole step's device time (its kernels overlap on two streams);
        # the sum of its kernels' times where no step record exists
        if ("step", d) in steps_by:
            ms = statistics.mean(steps_by[("step", d)])
        else:
            ms = sum(statistics.mean(v) for k, v in by.items() if k[1] == d)
        # the default pass runs steps d >= 2 as one launch that reads each
        # record once; the cage step, depth 1 and the exact pass read the
        # records again in a separate vertex pass
        fused = d >= 2 and not args.deterministic
        nb = metrics.level_bytes(levels[d], levels[d + 1], rec_bytes, subd.record_words == 4, d == 0, w.cage.U,
                                 topology=not points_op, fused=fused)
        per_depth.append({"depth": d + 1, "ms": ms, "refined_halfedges": levels[d + 1]["H"],
                          "halfedges_per_s": levels[d + 1]["H"] / (ms / 1e3), "alg_bytes": nb,
                          "gbs": nb / (ms / 1e3) / 1e9, "frac_of_peak": nb / (ms / 1e3) / 1e9 / peak})

    # adjoint of the same workload (points of every depth -> cage points),
    # through the C ABI on the subd's stream
    adj = adjoint_timing(subd, w, stream, flush, args.steps, torch, peak)

    # end to end through the C ABI with host buffers
    host_pts = torch.from_numpy(w.cage.vertex_points.copy()).pin_memory()
    e2e_ms = []
    torch.cuda.synchronize()
    if points_op:
        # the points of every depth from pinned cage points to pinned host
        # memory through the differentiable entry point (RefinePointsDevice)
        from halfedgecatmullclark_b200.torch_ext import refine_points
        host_out = torch.empty((subd.cumV, 3), dtype=torch.float32).pin_memory()
    for _ in range(args.e2e_steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        if points_op:
            with torch.cuda.stream(stream):
                x = host_pts.to("cuda", non_blocking=True)
                host_out.copy_(refine_points(x, subd), non_blocking=True)
        else:
            subd.upload_cage_points(host_pts.numpy())
            subd.refine_scatter()
            subd.download()
        b.record(stream)
        torch.cuda.synchronize()
        e2e_ms.append(a.elapsed_time(b))
    e2e_total = max_over_ranks(sum(e2e_ms), world)
    h2d = 12 * w.cage.V
    if points_op:
        d2h = 12 * subd.cumV
    else:
        d2h = 4 * subd.record_words * subd.cumH + 12 * subd.cumC + 12 * subd.cumV
    launches = len([r for r in recs if r["kernel"] not in ("clear", "step")]) // max(1, args.steps)

    base = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        try:
            base = cpu_reference(w, args.cpu_seconds, op=args.op)
        except Exception as exc:  # a missing baseline must not hide the GPU number
            base = {"value": None, "unit": UNIT, "cores": os.cpu_count(), "kind": "unavailable",
                    "sample": "error: %s" % exc}
    subd.close()
    del flush
    torch.cuda.empty_cache()
    # the batched workload (many uneven cages, forward + adjoint against a
    # loop of single-mesh calls), on the same line so that every run records it
    batch = None
    if not args.no_batch and not args.deterministic and args.op == "refine" and args.workload == "mixed_torus":
        batch = batch_measure(args, rank, world)
    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": config_dict(w, {"parallelism": "replicas x%d" % world,
                                      "deterministic": bool(args.deterministic), "op": args.op,
                                      "refined_halfedges_per_step": SH}),
            "e2e": {"value": world * SH * args.e2e_steps / (e2e_total / 1e3), "unit": UNIT,
                    "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "ms_per_step": e2e_total / args.e2e_steps},
            "gpu_launches": launches * args.steps,
            "roofline": {"bound": "hbm", "kernel": "%s@depth%d" % (dom_key[0], dom_key[1]),
                         "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                         "peak_kind": peak_kind, "alg_bytes_per_launch": dom_bytes,
                         "launch_ms": dom_ms,
                         "traffic": traffic},
            "per_depth": per_depth,
            "kernels": kernels[:12],
            "adjoint": adj,
            "clocks": clocks,
            "wall_s": wall,
        }
        if base is not None:
            line["cpu_baseline"] = base
        if batch is not None:
            line["batch"] = batch
        print(json.dumps(line))
    if world > 1:
        import torch.distributed as dist
        dist.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())

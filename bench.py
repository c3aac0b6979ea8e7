#!/usr/bin/env python3
"""Benchmark of the B200 volumetric estimator stage (PP3D + PB2D + BB1D with UPBP MIS).

One step = one UPBP iteration's estimator stage: build of the PP3D hash grid, the PB2D photon LBVH
and the BB1D beam LBVH, then the batched evaluation of every recorded camera-segment query
(evalBre + evalBeamBeamEstimate) and camera medium-vertex query (HashGrid::Process), splatted
into the framebuffer.  Units are queries (segment queries + point queries).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--config cube1024]

The headline arm is the batched mixed-precision stage.  On one GPU the same line also times, on the
same workload, the plain FP32 stage with the same warp-cooperative kernels (autotuned on its own),
the plain FP32 drop-in (one thread per query), and the mixed stage with B-P2D on, each with its
image rel-L2 against the GPU FP64 mode; and it checks a sample of the queries against the
reference's own estimators (``parity``).

On one GPU with the default workload the line also carries ``secondary_configs``: short runs of
configuration 2 (``boxes3``: the fused persistent kernel replayed as a CUDA graph against
per-estimator launches), configuration 3 (``beamstress``: mixed, plain FP32 and FP64, per-query
error percentiles against FP64) and configuration 4 (``diff512``: forward and adjoint times, device
memory, the adjoint against central differences of the FP64 forward).

Multi-GPU: ``--gpus N`` without a launcher starts N ranks itself (torch.distributed.run, one rank
per GPU, NCCL).  ``--shard queries`` (the default for N > 1): every rank builds the same structures
over the whole iteration and evaluates its pixel tiles of the queries, and one framebuffer
all-reduce per step combines them (strong scaling: one iteration gets faster).  ``--shard
iterations``: every rank evaluates its own iterations (weak scaling, as the reference runs one
renderer per thread over independent iterations).

Prints ONE JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import math
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "estimator queries/s and ms/iteration, batched mixed vs plain FP32, at rel L2<=1e-3"
FALLBACK_HBM_GBS = 6650.0

# Algorithmic bytes (per query and per accepted candidate), independent of the acceleration
# structure: query record 64 + camera MIS context 32 + output 12; BB1D candidate 72; PB2D/PP3D 52.
BYTES_PER_QUERY = 108
BYTES_PER_BB1D = 72
BYTES_PER_POINT_CAND = 52


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=6)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--config", default="cube1024")
    ap.add_argument("--mode", default="mixed", choices=["mixed", "plain"])
    ap.add_argument("--iterations", type=int, default=2, help="distinct iteration workloads cycled per rank")
    ap.add_argument("--cpu-seconds", type=float, default=12.0, help="CPU work per reference sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-accuracy", action="store_true", help="skip the image rel-L2 check against the FP64 mode")
    ap.add_argument("--no-device-passes", action="store_true",
                    help="skip the iteration traced on the device (light + camera passes, build, evaluate)")
    ap.add_argument("--no-autotune", action="store_true", help="keep the library's default tuning")
    ap.add_argument("--tuning", default=None,
                    help='fixed tuning instead of the autotuner, JSON (e.g. \'{"bb1d_leaf": 8, "beam_piece_radii": 6}\')')
    ap.add_argument("--no-graph", action="store_true", help="direct calls instead of the captured CUDA graph")
    ap.add_argument("--adjoint", action="store_true",
                    help="time forward + adjoint (dL/d sigma_a, sigma_s, g) of an L2 image loss instead")
    ap.add_argument("--shard", default=None, choices=["queries", "iterations"],
                    help="multi-GPU work split (default: queries when N > 1)")
    ap.add_argument("--no-arms", action="store_true",
                    help="skip the plain FP32, drop-in and B-P2D comparison arms (one GPU only)")
    ap.add_argument("--no-secondary", action="store_true",
                    help="skip the short runs of the other configurations (boxes3, beamstress, diff512)")
    ap.add_argument("--no-parity", action="store_true",
                    help="skip the check of sampled queries against the reference's estimators")
    ap.add_argument("--dropin", action="store_true",
                    help="the plain FP32 drop-in: thread-per-query BB1D gather, plain mode, leaves of 2 and 3 r "
                         "pieces (the best of a leaf / piece sweep for that gather on cube512)")
    ap.add_argument("--knn", default=None, metavar="PB2D,BB1D",
                    help="KNN radii: photons and beam origins per search (-r_initial_pb2d_knn, "
                         "-r_initial_bb1d_knn), found by the reference's kd-tree search")
    ap.add_argument("--bb1d-grid", type=int, default=0,
                    help="BB1D over the reference's uniform beam grid of this resolution (-gridres) instead of the "
                         "LBVH of beam pieces; keeps the library's tuning and skips the e2e, accuracy, device-pass, "
                         "comparison-arm, parity and secondary measurements, which are defined for the LBVH path")
    a = ap.parse_args()
    if a.bb1d_grid:
        a.no_autotune = a.no_e2e = a.no_accuracy = a.no_device_passes = a.no_arms = a.no_parity = True
        a.no_secondary = True
    if a.dropin:
        a.mode, a.no_autotune = "plain", True
        t = dict(DROPIN_TUNING)
        t.update(json.loads(a.tuning) if a.tuning else {})
        a.tuning = json.dumps(t)
    return a


# The plain FP32 drop-in: one thread per query for PB2D and BB1D, plain mode, leaves of 2 and 3 r
# pieces (the best of a leaf / piece sweep for the thread-per-query BB1D gather on cube512).
DROPIN_TUNING = {"bb1d_kernel": 0, "pb2d_kernel": 0, "bb1d_leaf": 2, "beam_piece_radii": 3.0}
UPBP_BP2D = 65536

# The reference CPU timings (the CPU baseline of the GPU arm and the --impl reference arm) use the
# same deterministic stratified sample: every S-th query (segment and point queries alike) with S
# chosen from the workload size so that one sample holds about REF_SAMPLE_QUERIES queries, and
# sample k of n starting at offset k*S//n.  Each sample's time x S + the per-thread build time
# extrapolates one whole iteration; the median over the samples is reported with its spread.
REF_SAMPLE_QUERIES = 12000


def dist_env():
    return int(os.environ.get("RANK", 0)), int(os.environ.get("WORLD_SIZE", 1)), int(os.environ.get("LOCAL_RANK", 0))


def workload_desc(cfg) -> dict:
    return {
        "workload": "%s: %dx%d, %d light sub-paths/iteration, max path length %d, radius %g, %s query beams, "
                    "%s photon beams%s" % (
                        cfg.name, cfg.width, cfg.height, cfg.light_paths, cfg.max_path_length, cfg.radius,
                        "LONG" if cfg.query_beam_type == 2 else "SHORT", "LONG" if cfg.photon_beam_type == 2 else "SHORT",
                        (" capped at %g" % cfg.beam_length_cap) if math.isfinite(cfg.beam_length_cap) else ""),
        "estimators": "PP3D+PB2D+BB1D with UPBP MIS (BPT|SURF|PP3D|PB2D|BB1D weights)",
        "l2_flush": "inputs larger than L2 (each iteration's records exceed 126 MB; iterations alternate)",
    }


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as fh:
            return float(json.load(fh)["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "--query-gpu=" + self.FIELDS, "--format=csv,noheader,nounits",
                                          "-i", str(self.device), "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self) -> dict:
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        time.sleep(0.25)
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, smax, power, reasons = [], [], [], set()
        names = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")
        for line in self.lines:
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
                power.append(float(parts[3]))
            except ValueError:
                continue
            for n, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "power_w_max": max(power) if power else None, "samples": len(sm), "reasons": sorted(reasons)}


def pinned_copy(w):
    """Copies of the workload arrays in page-locked host memory (for the end-to-end timing)."""
    import torch
    out = {}
    for k, v in w.items():
        if v.dtype.names is not None:
            raw = np.ascontiguousarray(v).view(np.uint8)
            t = torch.from_numpy(raw.copy()).pin_memory()
            out[k] = t.numpy().view(v.dtype).reshape(v.shape)
        else:
            t = torch.from_numpy(np.ascontiguousarray(v).copy()).pin_memory()
            out[k] = t.numpy()
    return out


def input_bytes(w) -> int:
    return int(sum(v.nbytes for k, v in w.items() if k not in ("params", "media")))


def kernel_source_hash() -> str:
    """Digest of the kernel sources that the committed ncu traffic figure belongs to."""
    import hashlib
    h = hashlib.sha256()
    csrc = os.path.join(ROOT, "smallupbp_b200", "csrc")
    for f in ("upbp_gather.cu", "upbp_device.cuh", "upbp_traverse.cuh", "upbp_kernels.cuh", "upbp_build.cu",
              "upbp_capi.cu"):
        with open(os.path.join(csrc, f), "rb") as fh:
            h.update(fh.read())
    return h.hexdigest()[:16]


def make_stages(works, dev, mode, stream, tuning=None, bb1d_grid=0):
    from smallupbp_b200 import abi, engine
    stages, structs = [], []
    for w in works:
        st = engine.EstimatorStage(dev, mode)
        st.set_stream(stream.cuda_stream)
        s = abi.make_structs(w)
        st.load(w, s)
        st.set_queries(w, s)
        if tuning:
            st.set_tuning(**tuning)
        if bb1d_grid:
            st.set_bb1d_grid(bb1d_grid)
        stages.append(st)
        structs.append(s)
    return stages, structs


def tune_stages(stages, structs, stream):
    import torch
    from smallupbp_b200 import autotune
    t0 = time.time()
    with torch.cuda.stream(stream):
        best, rep = autotune.autotune(stages[0], structs[0][0])
    for st in stages[1:]:
        st.set_tuning(**best)
    return {"best": best, "autotuned": True, "trials": rep["trials"], "seconds": time.time() - t0}


def time_stages(stages, units, steps, warmup, stream, graph, world, img_t, dev, clocks=False):
    """Warm-up, then `steps` timed steps (CUDA events on the library's stream; barrier and
    synchronize on both sides; max over ranks).  A step is clear + build + evaluate of the next
    iteration's stage, replayed as its CUDA graph after the warm-up, plus the framebuffer
    all-reduce when world > 1."""
    import torch
    from smallupbp_b200 import engine, multi
    n_iter = len(stages)
    graphs = set()

    def step(i):
        st = stages[i % n_iter]
        if id(st) in graphs:
            st.launch_graph()
        else:
            st.build()
            st.clear_image()
            st.evaluate()
        if world > 1:
            import torch.distributed as dist
            st.read_image_into(img_t.data_ptr())
            with torch.cuda.stream(stream):
                dist.all_reduce(img_t)

    with torch.cuda.stream(stream):
        for i in range(warmup):
            step(i)
        if graph:
            for st in stages:
                try:
                    st.capture_graph()
                except engine.UpbpError:  # not evaluated during the warm-up
                    st.build(); st.clear_image(); st.evaluate()
                    st.capture_graph()
                graphs.add(id(st))
    torch.cuda.synchronize()
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    torch.cuda.synchronize()
    sampler = ClockSampler(dev) if clocks else None
    if sampler:
        sampler.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    kern = {"build_ms": [], "pp3d_ms": [], "pb2d_ms": [], "bb1d_ms": []}
    launches, done = [], 0
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for i in range(steps):
            step(i)
            st = stages[i % n_iter]
            for k, v in st.timings().items():
                kern[k].append(v)
            b, e = st.launch_counts()
            launches.append(b + e)
            done += units[i % n_iter]
        ev1.record(stream)
    torch.cuda.synchronize()
    clock = sampler.stop() if sampler else None
    ms = ev0.elapsed_time(ev1)
    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        ms = multi.max_over_ranks(ms, "cuda")
        done = int(multi.sum_over_ranks(done, "cuda"))
    return {"ms": ms, "units": done, "value": done / (ms / 1000.0), "ms_per_step": ms / steps,
            "kernels_ms": {k: statistics.mean(v) for k, v in kern.items()}, "launches": int(sum(launches)),
            "clocks": clock}


def evaluate_once(st):
    """Per-query results and the image of one evaluation (outside any timed region)."""
    st.build()
    st.clear_image()
    st.evaluate()
    pb2d, bb1d = st.segment_results()
    return {"stats": st.query_stats(), "pb2d": pb2d, "bb1d": bb1d, "pp3d": st.point_results(),
            "image": st.image().astype(np.float64)}


def rel_l2(a, b) -> float:
    return float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))


def fp64_image(w, dev, stream, tuning):
    import torch
    from smallupbp_b200 import engine
    with torch.cuda.stream(stream), engine.EstimatorStage(dev, engine.MODE_FP64) as st:
        st.set_stream(stream.cuda_stream)
        st.set_tuning(**tuning)
        st.run(w)
        return st.image().astype(np.float64), st.query_stats()


def run_b200(args, cfg, rank, world, local_rank):
    import torch
    from smallupbp_b200 import abi, engine, multi, workload as W

    torch.cuda.set_device(local_rank)
    dev = local_rank
    shard = args.shard or ("queries" if world > 1 else "iterations")
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    mode = engine.MODE_MIXED if args.mode == "mixed" else engine.MODE_PLAIN
    n_iter = max(1, min(args.iterations, args.steps))
    t0 = time.time()
    works = []
    if shard == "queries":
        # every rank: the same iterations, its pixel tiles of their queries
        for it in range(n_iter):
            works.append(multi.shard_workload(W.make(cfg, iteration=it), cfg.width, rank, world))
    else:
        for it in multi.rank_iterations(rank, world, n_iter):
            works.append(W.make(cfg, iteration=it))
    gen_s = time.time() - t0
    stream = torch.cuda.Stream(device=dev)
    npix = cfg.width * cfg.height
    img_t = torch.zeros(npix * 3, dtype=torch.float32, device="cuda")
    stages, all_structs = make_stages(works, dev, mode, stream, json.loads(args.tuning) if args.tuning else None,
                                      args.bb1d_grid)
    tuning = {"best": {k: getattr(stages[0].get_tuning(), k) for k, _ in abi.Tuning._fields_}, "autotuned": False}
    if not args.no_autotune and not args.tuning:
        tuning = tune_stages(stages, all_structs, stream)
    units = [len(w["sq_path_length"]) + len(w["pq_path_length"]) for w in works]
    head = time_stages(stages, units, args.steps, args.warmup, stream, not args.no_graph, world, img_t, dev,
                       clocks=True)
    head["tuning"] = tuning["best"]
    ms_max, value = head["ms"], head["value"]

    # candidate statistics and per-query results (outside the timed region)
    res0 = evaluate_once(stages[0])
    stats = res0["stats"]
    nq, npq = len(works[0]["sq_path_length"]), len(works[0]["pq_path_length"])
    acc = {k: int(stats["count_" + k].astype(np.int64).sum()) for k in ("pb2d", "bb1d", "pp3d")}
    tested = stages[0].tested_counts()
    alg = {"pp3d": BYTES_PER_QUERY * npq + BYTES_PER_POINT_CAND * acc["pp3d"],
           "pb2d": BYTES_PER_QUERY * nq + BYTES_PER_POINT_CAND * acc["pb2d"],
           "bb1d": BYTES_PER_QUERY * nq + BYTES_PER_BB1D * acc["bb1d"]}
    avg = head["kernels_ms"]
    if tuning["best"].get("bb1d_kernel", 1) >= 3:
        # one persistent kernel evaluates PB2D and BB1D: its phase (bb1d_ms) carries both
        alg["bb1d"] += alg.pop("pb2d")
        alg["pb2d"] = 0
    dom = max(("pp3d", "pb2d", "bb1d"), key=lambda k: avg[k + "_ms"])
    peak, peak_kind = measured_peak()
    achieved = alg[dom] / (avg[dom + "_ms"] / 1000.0) / 1e9 if avg[dom + "_ms"] > 0 else None
    traffic, traffic_note = None, "no ncu capture committed for this kernel and workload"
    tfile = os.path.join(ROOT, "profiles", "traffic_%s_%s.json" % (dom, cfg.name))
    if args.bb1d_grid or args.knn:
        traffic_note = "no ncu traffic figure committed for this path (%s)" % (
            "BB1D over the reference grid" if args.bb1d_grid else "KNN radii")
    elif os.path.exists(tfile):
        try:
            with open(tfile) as fh:
                tj = json.load(fh)
            same_tuning = all(tuning["best"].get(k) == v for k, v in (tj.get("tuning") or {}).items())
            if tj.get("kernel_source_hash") == kernel_source_hash() and same_tuning:
                traffic = tj.get("dram_bytes_per_launch")
                traffic_note = tj.get("how", "")
            else:
                traffic_note = "the committed ncu capture is of other kernel sources or another tuning: not used"
        except Exception:
            traffic = None

    # end to end through the public API from page-locked host buffers.  Two contexts on two
    # streams take the steps in turn, so that a step's uploads (on its context's stream) overlap
    # the previous step's evaluation; every step still uploads all its inputs and reads its image
    # back inside the timed region.
    e2e = None
    if not args.no_e2e:
        pw = pinned_copy(works[0])
        streams = [stream, torch.cuda.Stream(device=dev)]
        ctxs = []
        for k in range(2):
            st = engine.EstimatorStage(dev, mode)
            st.set_stream(streams[k].cuda_stream)
            st.set_tuning(**tuning["best"])
            ctxs.append(st)
        host_img = torch.empty(npix * 3, dtype=torch.float32).pin_memory()
        s = abi.make_structs(pw)
        e_units = units[0]

        def e2e_steps(n):
            prev = None
            for k in range(n):
                st = ctxs[k % 2]
                with torch.cuda.stream(streams[k % 2]):
                    st.load(pw, s); st.set_queries(pw, s); st.build(); st.clear_image(); st.evaluate()
                if prev is not None:
                    prev.read_image_into(host_img.data_ptr())
                prev = st
            prev.read_image_into(host_img.data_ptr())

        e2e_steps(max(2, args.warmup))
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(streams[0])
        streams[1].wait_event(e0)
        e2e_steps(args.steps)
        streams[0].wait_stream(streams[1])
        e1.record(streams[0])
        torch.cuda.synchronize()
        e_ms = e0.elapsed_time(e1)
        e_units_total = e_units * args.steps
        if world > 1:
            e_ms = multi.max_over_ranks(e_ms, "cuda")
            e_units_total = int(multi.sum_over_ranks(e_units_total, "cuda"))
        e2e = {"value": e_units_total / (e_ms / 1000.0), "unit": "queries/s",
               "h2d_bytes_per_step": input_bytes(works[0]), "d2h_bytes_per_step": npix * 3 * 4,
               "ms_per_step": e_ms / args.steps,
               "pipeline": "two contexts alternate; a step's uploads overlap the previous step's evaluation"}
        for st in ctxs:
            st.close()

    # accuracy of every arm on the benchmark workload: image rel-L2 against the GPU FP64 mode (the
    # same candidates, all geometry, contributions and MIS weights in FP64)
    img64 = None
    accuracy = None
    if not args.no_accuracy:
        img64, stats64 = fp64_image(works[0], dev, stream, tuning["best"])
        l2 = rel_l2(res0["image"], img64)
        accuracy = {"image_rel_l2_vs_fp64": l2, "bound": 1e-3, "within_bound": l2 <= 1e-3,
                    "same_bb1d_candidates": bool(np.array_equal(stats["count_bb1d"], stats64["count_bb1d"]) and
                                                 np.array_equal(stats["hash_bb1d"], stats64["hash_bb1d"]))}

    # whole iteration on the device: light and camera passes, build, evaluate, image read back
    device_passes = None
    if not args.no_device_passes and cfg.name != "beamstress" and shard == "iterations":
        device_passes = run_device_passes(args, cfg, dev, mode, stream, tuning, npix, rank, world)
    for st in stages:
        st.close()

    # the comparison arms of the metric, on the same workload (one GPU)
    arms = plain_res = None
    if world == 1 and not args.no_arms and args.mode == "mixed" and not args.tuning:
        arms, plain_res = run_arms(args, works, units, dev, stream, img_t, head, res0, img64)

    parity = None
    if rank == 0 and world == 1 and not args.no_parity:
        checked = {args.mode: res0}
        if plain_res is not None:
            checked["plain"] = plain_res
        parity = reference_parity(works[0], checked)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(works[0], args.cpu_seconds)

    secondary = None
    if world == 1 and not args.no_secondary and cfg.name == "cube1024":
        secondary = run_secondary(dev, stream)

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
        dist.destroy_process_group()
    if rank != 0:
        return None
    line = {
        "metric": METRIC,
        "value": value,
        "unit": "queries/s",
        "n_gpus": world,
        "steps": args.steps,
        "warmup": args.warmup,
        "ms_per_step": ms_max / args.steps,
        "higher_is_better": True,
        "scaling": "strong" if shard == "queries" and world > 1 else "weak",
        "vs_baseline": None,
        "dtype": "f32" if args.mode == "plain" else "f32+f64",
        "data": "synthetic: seeded UPBP light/camera passes (Philox) in the %s scene; no dataset" % cfg.name,
        "config": dict(workload_desc(cfg), mode=args.mode + (" drop-in (thread per query)" if args.dropin else ""),
                       iterations_cycled=n_iter,
                       queries_per_iteration={"segment": nq, "point": npq},
                       photons=int((works[0]["lv_flags"] & 1).sum()), beams=len(works[0]["beam_length"]),
                       parallelism=("dp%d: each rank builds the iteration's structures and evaluates its 32x32 pixel "
                                    "tiles of the queries; framebuffer all-reduce" % world) if shard == "queries" else
                                   ("dp%d: one iteration per rank, framebuffer all-reduce" % world),
                       candidate_sets=("the reference's default grid evaluator (USE_GRID, Grid.hxx) at -gridres %d: "
                                       "its cells, cell lists and DDA walk" % args.bb1d_grid) if args.bb1d_grid else
                                      ("the reference's brute-force BB1D estimator (PhBrute.hxx) under the reach rule "
                                       "(FP64 segment distance <= r(u) + 2e-5 + 1e-3 r); the reference's default grid "
                                       "(USE_GRID) differs where a closest approach falls on a DDA cell boundary"),
                       tuning=tuning, cuda_graph=not args.no_graph),
        "ms_per_iteration": ms_max / args.steps,
        "kernels_ms": avg,
        "accepted_candidates": acc,
        "tested_candidates": tested,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                     "unit": "GB/s", "frac": achieved / peak if achieved is not None else None, "traffic": traffic,
                     "traffic_note": traffic_note, "algorithmic_bytes_per_launch": alg[dom]},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": head["launches"],
        "clocks": head["clocks"],
        "generate_s": gen_s,
        "device_passes": device_passes,
        "accuracy": accuracy,
        "arms": arms,
        "parity": parity,
        "secondary_configs": secondary,
    }
    return line


def run_secondary(dev, stream):
    """The other benchmark configurations, timed briefly in the same run (3 timed evaluations after a
    warm-up, CUDA events on the library's stream, the library's default tuning):

    * configuration 2 (`boxes3`, traced on the device): the fused persistent kernel for all camera
      segments replayed as a CUDA graph against per-estimator launches without a graph, mixed mode;
    * configuration 3 (`beamstress`): mixed, plain FP32 and FP64 modes, with the per-query relative
      error of mixed and plain against FP64 (percentiles) and the image rel-L2;
    * configuration 4 (`diff512`): forward (mixed) and adjoint of the L2 loss against the target
      medium, their times, the device memory, and the adjoint against central differences (step 1e-3)
      of the FP64 forward;
    * the reference's uniform beam grid at -gridres 64 on cube1024 (mixed), against the LBVH over
      beam pieces: build and BB1D times, accepted pairs, image rel-L2 between the two."""
    import torch
    from smallupbp_b200 import engine, workload as W

    def timed(st, fn, n=3):
        with torch.cuda.stream(stream):
            fn()
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(n):
                fn()
            e1.record(stream)
        torch.cuda.synchronize()
        return e0.elapsed_time(e1) / n

    out = {}
    # configuration 2
    cfg = W.config("boxes3")
    c2 = {}
    for name, tun, graph in (("fused_persistent_graph", {"bb1d_kernel": 4}, True),
                             ("per_estimator_launches", {"bb1d_kernel": 2}, False)):
        with torch.cuda.stream(stream):
            st = engine.EstimatorStage(dev, engine.MODE_MIXED)
            st.set_stream(stream.cuda_stream)
            st.set_tuning(**tun)
            st.trace(cfg, 0)
            st.build(); st.clear_image(); st.evaluate()
            queries = st.input_bytes("sq_pixel") // 4 + st.input_bytes("pq_pixel") // 4
            if graph:
                st.capture_graph()
                ms = timed(st, st.launch_graph)
            else:
                ms = timed(st, lambda: (st.build(), st.clear_image(), st.evaluate()))
            c2[name] = {"ms_per_iteration": ms, "queries_per_s": queries / (ms / 1000.0), "tuning": tun}
            st.close()
    c2["queries_per_iteration"] = int(queries)
    out["boxes3"] = c2
    # configuration 3
    w = W.make(W.config("beamstress"))
    res = {}
    for name, mode in (("mixed", engine.MODE_MIXED), ("plain_fp32", engine.MODE_PLAIN), ("fp64", engine.MODE_FP64)):
        with torch.cuda.stream(stream):
            st = engine.EstimatorStage(dev, mode)
            st.set_stream(stream.cuda_stream)
            st.run(w)
            ms = timed(st, lambda: (st.clear_image(), st.evaluate()))
            _, bb1d = st.segment_results()
            res[name] = {"ms": ms, "bb1d": bb1d.astype(np.float64), "image": st.image().astype(np.float64),
                         "count": st.query_stats()["count_bb1d"]}
            st.close()
    ref = res["fp64"]
    c3 = {"queries": len(w["sq_path_length"]), "beams": len(w["beam_length"]),
          "fp64_ms": ref["ms"], "accepted_pairs": int(ref["count"].astype(np.int64).sum())}
    # per query: the largest channel difference over the largest channel of the FP64 result, with a
    # floor of 1e-6 of the largest query so that near-zero queries do not dominate the percentiles
    qmax = np.abs(ref["bb1d"]).max(axis=1)
    nz = qmax > 0
    floor = 1e-6 * float(qmax.max()) if qmax.size else 0.0
    for name in ("mixed", "plain_fp32"):
        r = res[name]
        err = (np.abs(r["bb1d"] - ref["bb1d"]).max(axis=1) / np.maximum(qmax, floor))[nz]
        c3[name] = {"ms": r["ms"], "same_candidates": bool(np.array_equal(r["count"], ref["count"])),
                    "image_rel_l2_vs_fp64": rel_l2(r["image"], ref["image"]),
                    "per_query_rel_err_vs_fp64": {q: float(np.percentile(err, p)) for q, p in
                                                  (("p50", 50), ("p99", 99), ("p99.9", 99.9), ("max", 100))}
                    if err.size else None}
    out["beamstress"] = c3
    # the reference's uniform beam grid (upbp_set_bb1d_grid) on the headline workload at -gridres
    # 64, the resolution of the CPU baseline: build + evaluate against the LBVH over beam pieces
    cfg = W.config("cube1024")
    cg = {"grid_res": 64}
    for name, grid in (("lbvh_pieces", None), ("reference_grid", 64)):
        with torch.cuda.stream(stream):
            st = engine.EstimatorStage(dev, engine.MODE_MIXED)
            st.set_stream(stream.cuda_stream)
            if grid:
                st.set_bb1d_grid(grid)
            st.trace(cfg, 0)
            st.build(); st.clear_image(); st.evaluate()
            ms = timed(st, lambda: (st.build(), st.clear_image(), st.evaluate()))
            t = st.timings()
            cg[name] = {"ms_per_iteration": ms, "build_ms": t["build_ms"], "bb1d_ms": t["bb1d_ms"],
                        "accepted_pairs": int(st.query_stats()["count_bb1d"].astype(np.int64).sum()),
                        "image": st.image().astype(np.float64)}
            st.close()
    cg["image_rel_l2_grid_vs_pieces"] = rel_l2(cg["reference_grid"].pop("image"), cg["lbvh_pieces"].pop("image"))
    out["cube1024_reference_grid"] = cg
    # KNN radii (-r_initial_pb2d_knn 8, -r_initial_bb1d_knn 6) on the headline workload: the
    # reference's own kd-tree search (the default) and the exact k-th nearest
    ck = {"pb2d_knn": 8, "bb1d_knn": 6}
    for name, exact in (("reference_search", 0), ("exact", 1)):
        cfg = W.config("cube1024")
        cfg.pb2d_knn, cfg.bb1d_knn = ck["pb2d_knn"], ck["bb1d_knn"]
        w = W.make(cfg)
        w["params"]["knn_exact"] = exact
        with torch.cuda.stream(stream):
            st = engine.EstimatorStage(dev, engine.MODE_MIXED)
            st.set_stream(stream.cuda_stream)
            st.run(w)
            ms = timed(st, lambda: (st.build(), st.clear_image(), st.evaluate()))
            t = st.timings()
            ck[name] = {"ms_per_iteration": ms, "build_ms": t["build_ms"], "bb1d_ms": t["bb1d_ms"],
                        "accepted_pairs": int(st.query_stats()["count_bb1d"].astype(np.int64).sum())}
            st.close()
    out["cube1024_knn_radii"] = ck
    # configuration 4
    w = W.make(W.config("diff512"))
    media = np.array(w["media"], copy=True)
    medium = 1

    def with_media(sa, ss, g):
        m = np.array(media, copy=True)
        m[medium]["absorption"], m[medium]["scattering"], m[medium]["mean_cosine"] = sa, ss, g
        return m

    with torch.cuda.stream(stream):
        fd = engine.EstimatorStage(dev, engine.MODE_FP64)
        fd.set_stream(stream.cuda_stream)
        fd.run(w)

        def image(m):
            fd.set_media(m)
            fd.clear_image()
            fd.evaluate()
            return fd.image().astype(np.float64)

        target = image(with_media((0.05,) * 3, (0.7,) * 3, 0.5))
        base = image(media)
        grad_img = torch.from_numpy((2.0 * (base - target)).astype(np.float32).reshape(-1)).cuda(dev)
        st = engine.EstimatorStage(dev, engine.MODE_MIXED)
        st.set_stream(stream.cuda_stream)
        st.run(w)
        torch.cuda.synchronize()
        fwd_ms = timed(st, lambda: (st.clear_image(), st.evaluate()))
        adj = st.adjoint(grad_img.data_ptr(), medium)
        adj_ms = timed(st, lambda: st.adjoint(grad_img.data_ptr(), medium))
        dev_bytes = st.device_bytes()
        st.close()
        m0 = media[medium]
        sa0, ss0, g0 = float(m0["absorption"][0]), float(m0["scattering"][0]), float(m0["mean_cosine"])
        h = 1e-3
        loss = lambda m: float(((image(m) - target) ** 2).sum())
        fds = {"sigma_a": (loss(with_media((sa0 + h,) * 3, (ss0,) * 3, g0)) -
                           loss(with_media((sa0 - h,) * 3, (ss0,) * 3, g0))) / (2 * h),
               "sigma_s": (loss(with_media((sa0,) * 3, (ss0 + h,) * 3, g0)) -
                           loss(with_media((sa0,) * 3, (ss0 - h,) * 3, g0))) / (2 * h),
               "g": (loss(with_media((sa0,) * 3, (ss0,) * 3, g0 + h)) - loss(with_media((sa0,) * 3, (ss0,) * 3, g0 - h))) / (2 * h)}
        fd.close()
    got = {"sigma_a": float(adj[0:3].sum()), "sigma_s": float(adj[3:6].sum()), "g": float(adj[6])}
    out["diff512"] = {"forward_ms": fwd_ms, "adjoint_ms": adj_ms, "device_bytes": int(dev_bytes),
                      "transmittance": "recomputed in the adjoint, not stored",
                      "grad_adjoint": got, "grad_central_differences_fp64": fds,
                      "max_rel_err": max(abs(got[k] - fds[k]) / max(abs(fds[k]), 1e-30) for k in got),
                      "bound": 1e-3}
    return out


def run_arms(args, works, units, dev, stream, img_t, head, res0, img64):
    """The metric's comparison on the same workload and in the same run: plain FP32 with the same
    warp-cooperative kernels (autotuned on its own), the plain FP32 drop-in (one thread per query),
    and the mixed stage with B-P2D on; each with its image rel-L2 against the FP64 mode."""
    from smallupbp_b200 import engine
    arms = {"mixed": {"ms_per_iteration": head["ms_per_step"], "value": head["value"],
                      "bb1d_ms": head["kernels_ms"]["bb1d_ms"],
                      "image_rel_l2_vs_fp64": rel_l2(res0["image"], img64) if img64 is not None else None}}
    plain_res = None
    for name, mode, tun, steps, warmup in (
            ("plain_fp32", engine.MODE_PLAIN, None, args.steps, args.warmup),
            ("dropin_fp32", engine.MODE_PLAIN, DROPIN_TUNING, min(args.steps, 2), 1)):
        stages, structs = make_stages(works, dev, mode, stream, tun)
        if tun:
            tuning = {"best": dict(tun), "autotuned": False}
        elif not args.no_autotune:
            tuning = tune_stages(stages, structs, stream)
        else:
            tuning = {"best": None, "autotuned": False}
        r = time_stages(stages, units, steps, warmup, stream, not args.no_graph, 1, img_t, dev)
        res = evaluate_once(stages[0])
        same = bool(np.array_equal(res["stats"]["count_bb1d"], res0["stats"]["count_bb1d"]) and
                    np.array_equal(res["stats"]["hash_bb1d"], res0["stats"]["hash_bb1d"]))
        arms[name] = {"ms_per_iteration": r["ms_per_step"], "value": r["value"], "steps": steps, "warmup": warmup,
                      "bb1d_ms": r["kernels_ms"]["bb1d_ms"], "tuning": tuning["best"],
                      "image_rel_l2_vs_fp64": rel_l2(res["image"], img64) if img64 is not None else None,
                      "same_candidates_as_mixed": same}
        if name == "plain_fp32":
            plain_res = res
        for st in stages:
            st.close()
    # B-P2D on (the fourth estimator; the reference has none, so the headline runs without it)
    wb = []
    for w in works:
        w2 = dict(w)
        w2["params"] = w["params"].copy()
        w2["params"]["techniques"] = int(w["params"]["techniques"][0]) | UPBP_BP2D
        wb.append(w2)
    stages, _ = make_stages(wb, dev, engine.MODE_MIXED, stream, head["tuning"])
    r = time_stages(stages, units, min(args.steps, 5), args.warmup, stream, not args.no_graph, 1, img_t, dev)
    for st in stages:
        st.close()
    arms["mixed_with_bp2d"] = {"ms_per_iteration": r["ms_per_step"], "value": r["value"],
                               "estimators": "PP3D+PB2D+BB1D+B-P2D (B-P2D standalone, MIS weight 1)"}
    m = arms["mixed"]["ms_per_iteration"]
    arms["speedup_mixed_vs_plain_fp32"] = arms["plain_fp32"]["ms_per_iteration"] / m
    arms["speedup_mixed_vs_dropin_fp32"] = arms["dropin_fp32"]["ms_per_iteration"] / m
    arms["target"] = "mixed >= 3x the plain FP32 GPU drop-in at image rel-L2 <= 1e-3 against FP64"
    return arms, plain_res


def reference_parity(w, results: dict) -> dict:
    """Sampled queries of the benchmark workload evaluated by the reference's own estimator code
    (EmbreeBre, the brute-force PhotonBeamsEvaluator, HashGrid + RangeQuery; oracle/_ref) and
    compared with the GPU's per-query candidate counts, candidate hashes and contributions: every
    S-th segment and point query, S chosen for about 2,000 segment queries."""
    from oracle import ref
    if not ref.available():
        return {"unavailable": "oracle/_ref not built on this machine"}
    t0 = time.time()
    nq, npq = len(w["sq_path_length"]), len(w["pq_path_length"])
    stride = max(1, nq // 2000)
    sess = ref.Session(w, ref.PB2D | ref.BB1D_BRUTE | ref.PP3D | ref.CANDIDATES, ref_threads())
    o = sess.eval_outputs(0, stride)
    sess.close()
    si, pi = np.arange(0, nq, stride), np.arange(0, npq, stride)
    out = {"queries_checked": {"segment": int(len(si)), "point": int(len(pi))}, "stride": stride,
           "reference": "PhotonBeamsEvaluator brute force (PhBrute.hxx), EmbreeBre, HashGrid/RangeQuery",
           "accepted_checked": {k: int(o["count_" + k][idx].astype(np.int64).sum())
                                for k, idx in (("pb2d", si), ("bb1d", si), ("pp3d", pi))}}
    want = {"pb2d": o["pb2d"], "bb1d": o["bb1d_brute"], "pp3d": o["pp3d"]}
    for name, res in results.items():
        if res is None:
            continue
        mism, rel = {}, {}
        for est, idx in (("pb2d", si), ("bb1d", si), ("pp3d", pi)):
            st = res["stats"]
            mism[est] = int(((st["count_" + est][idx] != o["count_" + est][idx]) |
                             (st["hash_" + est][idx] != o["hash_" + est][idx])).sum())
            g, r = res[est][idx].astype(np.float64), want[est][idx].astype(np.float64)
            floor = 1e-6 * max(float(np.abs(r).max()) if len(r) else 0.0, 1e-30)
            e = (np.abs(g - r) / (np.abs(r) + floor)).max(axis=1) if len(idx) else np.zeros(0)
            rel[est] = {"max_rel": float(e.max()) if len(e) else 0.0,
                        "within_1e-4": float((e <= 1e-4).mean()) if len(e) else 1.0}
        out[name] = {"candidate_mismatches": mism, "contributions": rel}
    out["seconds"] = time.time() - t0
    return out


def ref_threads() -> int:
    """Host threads for the reference: all cores, fewer when host memory cannot hold a copy of the
    structures per thread (about 5 GB each at cube1024)."""
    cores = os.cpu_count() or 1
    threads = cores
    try:
        with open("/proc/meminfo") as fh:
            avail_gb = int([l for l in fh if l.startswith("MemAvailable")][0].split()[1]) / 1e6
        threads = max(1, min(cores, int((avail_gb - 8) / 5.0)))
    except Exception:
        pass
    return threads


def reference_timing(w, samples: int, warmup: int, threads: int, stride_scale: int = 1) -> dict:
    """The reference's estimators (grid BB1D at -gridres 64) timed on the shared stratified sample:
    stride S (times stride_scale), sample k of `samples` at offset k*S//samples; each sample's
    time x S plus the per-thread build extrapolates one iteration, and the median is reported."""
    from oracle import ref
    ref.set_grid_options(64)
    sess = ref.Session(w, ref.PB2D | ref.BB1D_GRID | ref.PP3D, threads)
    total = sess.n_segment + sess.n_point
    S = max(1, int(round(total / REF_SAMPLE_QUERIES))) * stride_scale
    offs = [(k * S) // samples for k in range(samples)]
    for i in range(warmup):
        sess.eval(offs[i % samples], S)
    times = [sess.eval(o, S) for o in offs]
    sess.close()
    full = sorted(sess.build_ms + t * S for t in times)
    med = statistics.median(full)
    vals = [total / (f / 1000.0) for f in full]
    return {"value": total / (med / 1000.0), "ms_per_iteration": med, "build_ms": sess.build_ms,
            "sample_ms": [round(t, 1) for t in times], "median_sample_ms": statistics.median(times),
            "stride": S, "sampled_fraction": 1.0 / S, "samples": samples,
            "spread": {"min": min(vals), "max": max(vals)}}


def run_device_passes(args, cfg, dev, mode, stream, tuning, npix, rank, world):
    """Iterations traced on the device (upbp_trace_light_paths + upbp_trace_camera_paths), then
    built and evaluated, the framebuffer read back to page-locked host memory: the estimator
    stage with no host-side generation and no upload."""
    import torch
    from smallupbp_b200 import engine
    st = engine.EstimatorStage(dev, mode)
    st.set_stream(stream.cuda_stream)
    st.set_tuning(**tuning["best"])
    host_img = torch.empty(npix * 3, dtype=torch.float32).pin_memory()
    n_it = max(1, args.iterations)
    queries = []
    with torch.cuda.stream(stream):
        for i in range(max(1, args.warmup)):
            st.trace(cfg, rank + world * (i % n_it)); st.build(); st.clear_image(); st.evaluate()
            st.read_image_into(host_img.data_ptr())
        torch.cuda.synchronize()
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
        trace_ms = 0.0
        ev[0].record(stream)
        for i in range(args.steps):
            t0 = torch.cuda.Event(enable_timing=True)
            t1 = torch.cuda.Event(enable_timing=True)
            t0.record(stream)
            st.trace(cfg, rank + world * (i % n_it))
            t1.record(stream)
            st.build(); st.clear_image(); st.evaluate()
            st.read_image_into(host_img.data_ptr())
            queries.append(st._nq + st._np)
            torch.cuda.synchronize()
            trace_ms += t0.elapsed_time(t1)
        ev[1].record(stream)
    torch.cuda.synchronize()
    ms = ev[0].elapsed_time(ev[1])
    st.close()
    if world > 1:
        from smallupbp_b200 import multi
        ms = multi.max_over_ranks(ms, "cuda")
    from smallupbp_b200 import abi
    scene_bytes = ctypes.sizeof(abi.Scene) + ctypes.sizeof(abi.Params) + len(cfg.media) * ctypes.sizeof(abi.Medium)
    return {"value": sum(queries) * world / (ms / 1000.0), "unit": "queries/s", "ms_per_iteration": ms / args.steps,
            "trace_ms_per_iteration": trace_ms / args.steps, "h2d_bytes_per_step": scene_bytes,
            "d2h_bytes_per_step": npix * 3 * 4,
            "note": "light and camera sub-paths traced on the GPU (the host generator's records, bit for bit), "
                    "then build + evaluate; only the scene description and params cross from the host"}


def cpu_baseline(w, seconds: float) -> dict:
    """The reference estimator code (oracle/_ref, built from the reference sources) timed on this
    host's cores on the shared stratified sample (the same samples as --impl reference), median of
    five, plus the same code on one core."""
    from oracle import ref
    if not ref.available():
        return {"value": None, "unit": "queries/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built on this machine"}
    threads = ref_threads()
    r = reference_timing(w, 5, 1, threads)
    out = {"value": r["value"], "unit": "queries/s", "cores": threads, "kind": "reference",
           "sample": "reference SmallUPBP estimators (EmbreeBre + PhotonBeamsEvaluator USE_GRID -gridres 64 + "
                     "HashGrid/RangeQuery), one structure set per thread; 5 samples of every %d-th query (strata "
                     "k*%d/5), each %.1f s median, extrapolated linearly to the iteration plus the per-thread build "
                     "(%.1f s); median of the 5" % (r["stride"], r["stride"], r["median_sample_ms"] / 1000.0,
                                                   r["build_ms"] / 1000.0),
           "ms_per_iteration": r["ms_per_iteration"], "sampled_fraction": r["sampled_fraction"],
           "spread": r["spread"]}
    one = reference_timing(w, 3, 0, 1, stride_scale=16)
    out["one_core"] = {"value": one["value"], "unit": "queries/s", "ms_per_iteration": one["ms_per_iteration"],
                       "sample": "3 samples of every %d-th query on one thread (%.1f s each), plus its build (%.1f s); "
                                 "median" % (one["stride"], one["median_sample_ms"] / 1000.0, one["build_ms"] / 1000.0),
                       "spread": one["spread"]}
    return out


def run_reference(args, cfg, rank, world):
    """--impl reference: the reference's own CPU estimator code on this host's cores.  A step is one
    sample of the shared stratified sample (every S-th query; the samples take the strata
    k*S/steps), timed; the value extrapolates the median sample to the whole iteration, with the
    per-thread build.  Under torchrun only rank 0 works."""
    if rank != 0:
        return None
    from oracle import ref
    from smallupbp_b200 import workload as W
    if not ref.available():
        return {"impl": "reference", "unavailable": "oracle/_ref (reference built from its sources) is not present"}
    w = W.make(cfg, iteration=0)
    threads = ref_threads()
    r = reference_timing(w, max(1, args.steps), args.warmup, threads)
    value = r["value"]
    return {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": r["median_sample_ms"], "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "impl": "reference",
        "data": "synthetic: seeded UPBP light/camera passes (Philox) in the %s scene; no dataset" % cfg.name,
        "config": dict(workload_desc(cfg), grid_resolution=64),
        "ms_per_iteration": r["ms_per_iteration"],
        "steps_are": "samples: each step evaluates every %d-th query (%.4f of the iteration); ms_per_step is the "
                     "median sample's wall time, ms_per_iteration its extrapolation plus the per-thread build "
                     "(%.1f s)" % (r["stride"], r["sampled_fraction"], r["build_ms"] / 1000.0),
        "spread": r["spread"],
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": "reference",
                         "sample": "%d samples of every %d-th query (strata k*%d/%d), median extrapolated with the "
                                   "per-thread build (%.1f s)" % (args.steps, r["stride"], r["stride"], args.steps,
                                                                 r["build_ms"] / 1000.0)},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def run_adjoint(args, cfg, rank, world, local_rank):
    """Differentiable estimator: one step = forward (mixed mode) + adjoint of the L2 loss against a
    target rendered with sigma_s = 0.7, sigma_a = 0.05, g = 0.5 (from sigma_s = 0.5, sigma_a = 0.1,
    g = 0.3), gradients with respect to the grey sigma_a, sigma_s and g of the scene's medium."""
    import torch
    from smallupbp_b200 import autograd, engine, workload as W

    torch.cuda.set_device(local_rank)
    dev = torch.device("cuda", local_rank)
    w = W.make(cfg, iteration=rank)
    stream = torch.cuda.Stream(device=dev)
    st = engine.EstimatorStage(local_rank, engine.MODE_MIXED)
    st.set_stream(stream.cuda_stream)
    media = np.array(w["media"], copy=True)
    medium = 1
    units = len(w["sq_path_length"]) + len(w["pq_path_length"])

    def grey(v, grad=False):
        return torch.full((3,), v, dtype=torch.float64, device=dev, requires_grad=grad)

    with torch.cuda.stream(stream):
        st.run(w)
        torch.cuda.reset_peak_memory_stats(dev)
        tgt = autograd.render(st, media, medium, grey(0.05), grey(0.7), torch.tensor(0.5, dtype=torch.float64,
                                                                                       device=dev)).detach().clone()

        def step():
            sa, ss = grey(0.1, True), grey(0.5, True)
            g = torch.tensor(0.3, dtype=torch.float64, device=dev, requires_grad=True)
            e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
            e0.record(stream)
            img = autograd.render(st, media, medium, sa, ss, g)
            loss = ((img.double() - tgt.double()) ** 2).sum()
            e1.record(stream)
            loss.backward()
            e2.record(stream)
            return e0, e1, e2, (sa.grad.sum().item(), ss.grad.sum().item(), g.grad.item()), loss.item()

        for _ in range(args.warmup):
            step()
        torch.cuda.synchronize(dev)
        fwd, bwd = [], []
        ev_first = ev_last = None
        for _ in range(args.steps):
            e0, e1, e2, grads, loss = step()
            torch.cuda.synchronize(dev)
            fwd.append(e0.elapsed_time(e1))
            bwd.append(e1.elapsed_time(e2))
            ev_first = ev_first or e0
            ev_last = e2
        total_ms = ev_first.elapsed_time(ev_last)
    peak = st.device_bytes() + torch.cuda.max_memory_allocated(dev)
    st.close()
    if rank != 0:
        return None
    return {
        "metric": METRIC + " (forward + adjoint)", "value": units * args.steps / (total_ms / 1000.0), "unit": "queries/s",
        "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": total_ms / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32 (adjoint: f32 tangents, f64 accumulation)",
        "data": "synthetic: seeded UPBP light/camera passes (Philox) in the %s scene; no dataset" % cfg.name,
        "config": dict(workload_desc(cfg), mode="mixed forward + dual-number adjoint (FP32 tangents)",
                       loss="sum (I - I_target)^2, target sigma_s=0.7 sigma_a=0.05 g=0.5, at sigma_s=0.5 "
                            "sigma_a=0.1 g=0.3"),
        "adjoint": {"forward_ms": statistics.median(fwd), "backward_ms": statistics.median(bwd),
                    "peak_device_bytes": int(peak), "loss": loss,
                    "grad": {"sigma_a": grads[0], "sigma_s": grads[1], "g": grads[2]}},
    }


def spawn_ranks(n: int) -> int:
    """Start n ranks of this script (one per GPU) under torch.distributed.run on this node."""
    import socket
    with socket.socket() as sk:
        sk.bind(("127.0.0.1", 0))
        port = sk.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(n),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    args = parse()
    rank, world, local_rank = dist_env()
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        sys.exit(spawn_ranks(args.gpus))
    from smallupbp_b200 import workload as W
    cfg = W.config(args.config)
    if args.knn:
        cfg.pb2d_knn, cfg.bb1d_knn = (int(x) for x in args.knn.split(","))
    if args.impl == "reference":
        line = run_reference(args, cfg, rank, world)
    elif args.adjoint:
        line = run_adjoint(args, cfg, rank, world, local_rank)
    else:
        line = run_b200(args, cfg, rank, world, local_rank)
    if rank == 0 and line is not None:
        print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()

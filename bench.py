#!/usr/bin/env python3
"""Benchmark of the B200 volumetric estimator stage (PP3D + PB2D + BB1D with UPBP MIS).

One step = one UPBP iteration's estimator stage: build of the PP3D hash grid, the PB2D photon LBVH
and the BB1D beam LBVH, then the batched evaluation of every recorded camera-segment query
(evalBre + evalBeamBeamEstimate) and camera medium-vertex query (HashGrid::Process), splatted
into the framebuffer.  Units are queries (segment queries + point queries).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl b200|reference] [--config cube1024]

Multi-GPU (torchrun, one rank per GPU): every rank evaluates its own iterations (independent
seeds, as the reference runs one renderer per thread over independent iterations) and the
framebuffers are combined with one NCCL all-reduce per step: weak scaling.

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
    ap.add_argument("--dropin", action="store_true",
                    help="the plain FP32 drop-in: thread-per-query BB1D gather, plain mode, leaves of 2 and 3 r "
                         "pieces (the best of a leaf / piece sweep for that gather on cube512)")
    a = ap.parse_args()
    if a.dropin:
        a.mode, a.no_autotune = "plain", True
        t = {"bb1d_leaf": 2, "beam_piece_radii": 3.0}
        t.update(json.loads(a.tuning) if a.tuning else {})
        t["bb1d_kernel"] = 0
        a.tuning = json.dumps(t)
    return a


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


def run_b200(args, cfg, rank, world, local_rank):
    import torch
    from smallupbp_b200 import abi, engine, multi, workload as W

    torch.cuda.set_device(local_rank)
    dev = local_rank
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    mode = engine.MODE_MIXED if args.mode == "mixed" else engine.MODE_PLAIN
    n_iter = max(1, min(args.iterations, args.steps))
    t0 = time.time()
    works = []
    for it in multi.rank_iterations(rank, world, n_iter):
        works.append(W.make(cfg, iteration=it))
    gen_s = time.time() - t0
    stream = torch.cuda.Stream(device=dev)
    npix = cfg.width * cfg.height
    img_t = torch.zeros(npix * 3, dtype=torch.float32, device="cuda")
    stages, all_structs = [], []
    for w in works:
        st = engine.EstimatorStage(dev, mode)
        st.set_stream(stream.cuda_stream)
        s = abi.make_structs(w)
        st.load(w, s)
        st.set_queries(w, s)
        if args.tuning:
            st.set_tuning(**json.loads(args.tuning))
        stages.append(st)
        all_structs.append(s)
    tuning = {"best": {k: getattr(stages[0].get_tuning(), k) for k, _ in abi.Tuning._fields_}, "autotuned": False}
    if not args.no_autotune and not args.tuning:
        from smallupbp_b200 import autotune
        t_at = time.time()
        with torch.cuda.stream(stream):
            best, rep = autotune.autotune(stages[0], all_structs[0][0])
        for st in stages[1:]:
            st.set_tuning(**best)
        tuning = {"best": best, "autotuned": True, "trials": rep["trials"], "seconds": time.time() - t_at}
    units = [len(w["sq_path_length"]) + len(w["pq_path_length"]) for w in works]

    graphs = set()

    def step(i):
        st = stages[i % n_iter]
        if id(st) in graphs:
            st.launch_graph()  # clear + build + evaluate, captured after the warm-up
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
        for i in range(args.warmup):
            step(i)
        if not args.no_graph:
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
    clocks = ClockSampler(dev)
    clocks.start()
    ev0 = torch.cuda.Event(enable_timing=True)
    ev1 = torch.cuda.Event(enable_timing=True)
    kern = {"build_ms": [], "pp3d_ms": [], "pb2d_ms": [], "bb1d_ms": []}
    launches = []
    done_units = 0
    with torch.cuda.stream(stream):
        ev0.record(stream)
        for i in range(args.steps):
            step(i)
            st = stages[i % n_iter]
            for k2, v in st.timings().items():
                kern[k2].append(v)
            b, e = st.launch_counts()
            launches.append(b + e)
            done_units += units[i % n_iter]
        ev1.record(stream)
    torch.cuda.synchronize()
    clock = clocks.stop()
    ms = ev0.elapsed_time(ev1)
    # max over ranks, total units over ranks
    ms_max, units_total = ms, done_units
    if world > 1:
        ms_max = multi.max_over_ranks(ms, "cuda")
        units_total = int(multi.sum_over_ranks(done_units, "cuda"))
    value = units_total / (ms_max / 1000.0)

    # candidate statistics (outside the timed region) for the roofline
    st0 = stages[0]
    st0.build()
    st0.clear_image()
    st0.evaluate()
    stats = st0.query_stats()
    nq, npq = len(works[0]["sq_path_length"]), len(works[0]["pq_path_length"])
    acc = {k: int(stats["count_" + k].astype(np.int64).sum()) for k in ("pb2d", "bb1d", "pp3d")}
    tested = st0.tested_counts()
    alg = {"pp3d": BYTES_PER_QUERY * npq + BYTES_PER_POINT_CAND * acc["pp3d"],
           "pb2d": BYTES_PER_QUERY * nq + BYTES_PER_POINT_CAND * acc["pb2d"],
           "bb1d": BYTES_PER_QUERY * nq + BYTES_PER_BB1D * acc["bb1d"]}
    avg = {k: statistics.mean(v) for k, v in kern.items()}
    if tuning["best"].get("bb1d_kernel", 1) >= 3:
        # one persistent kernel evaluates PB2D and BB1D: its phase (bb1d_ms) carries both
        alg["bb1d"] += alg.pop("pb2d")
        alg["pb2d"] = 0
    dom = max(("pp3d", "pb2d", "bb1d"), key=lambda k: avg[k + "_ms"])
    peak, peak_kind = measured_peak()
    achieved = alg[dom] / (avg[dom + "_ms"] / 1000.0) / 1e9 if avg[dom + "_ms"] > 0 else None
    traffic = None
    tfile = os.path.join(ROOT, "profiles", "traffic_%s_%s.json" % (dom, cfg.name))
    if os.path.exists(tfile):
        try:
            with open(tfile) as fh:
                traffic = json.load(fh).get("dram_bytes_per_launch")
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
        if world > 1:
            e_ms = multi.max_over_ranks(e_ms, "cuda")
        e2e = {"value": e_units * args.steps * world / (e_ms / 1000.0), "unit": "queries/s",
               "h2d_bytes_per_step": input_bytes(works[0]), "d2h_bytes_per_step": npix * 3 * 4,
               "ms_per_step": e_ms / args.steps,
               "pipeline": "two contexts alternate; a step's uploads overlap the previous step's evaluation"}
        for st in ctxs:
            st.close()

    # accuracy of the measured mode on the benchmark workload: image rel-L2 against the FP64 mode
    # (the same candidates, all geometry, contributions and MIS weights in FP64)
    accuracy = None
    if not args.no_accuracy:
        accuracy = image_accuracy(works[0], dev, mode, tuning, stream)

    # whole iteration on the device: light and camera passes, build, evaluate, image read back
    device_passes = None
    if not args.no_device_passes and cfg.name != "beamstress":
        device_passes = run_device_passes(args, cfg, dev, mode, stream, tuning, npix, rank, world)

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline(works[0], args.cpu_seconds)

    if world > 1:
        import torch.distributed as dist
        dist.barrier()
    for st in stages:
        st.close()
    if world > 1:
        import torch.distributed as dist
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
        "scaling": "weak",
        "vs_baseline": None,
        "dtype": "f32" if args.mode == "plain" else "f32+f64",
        "data": "synthetic: seeded UPBP light/camera passes (Philox) in the %s scene; no dataset" % cfg.name,
        "config": dict(workload_desc(cfg), mode=args.mode + (" drop-in (thread per query)" if args.dropin else ""),
                       iterations_cycled=n_iter,
                       queries_per_iteration={"segment": nq, "point": npq},
                       photons=int((works[0]["lv_flags"] & 1).sum()), beams=len(works[0]["beam_length"]),
                       parallelism="dp%d (one iteration per rank, framebuffer all-reduce)" % world,
                       tuning=tuning, cuda_graph=not args.no_graph),
        "ms_per_iteration": ms_max / args.steps,
        "kernels_ms": avg,
        "accepted_candidates": acc,
        "tested_candidates": tested,
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak, "peak_kind": peak_kind,
                     "unit": "GB/s", "frac": achieved / peak if achieved is not None else None, "traffic": traffic,
                     "algorithmic_bytes_per_launch": alg[dom]},
        "cpu_baseline": cpu,
        "e2e": e2e,
        "gpu_launches": int(sum(launches)),
        "clocks": clock,
        "generate_s": gen_s,
        "device_passes": device_passes,
        "accuracy": accuracy,
    }
    return line


def image_accuracy(w, dev, mode, tuning, stream):
    """Image rel-L2 of `mode` against the GPU FP64 mode on workload `w` (one iteration)."""
    import torch
    from smallupbp_b200 import engine
    imgs, counts = {}, {}
    for m in (mode, engine.MODE_FP64):
        with torch.cuda.stream(stream), engine.EstimatorStage(dev, m) as st:
            st.set_stream(stream.cuda_stream)
            st.set_tuning(**tuning["best"])
            st.run(w)
            imgs[m] = st.image().astype(np.float64)
            counts[m] = int(st.query_stats()["count_bb1d"].astype(np.int64).sum())
    a, b = imgs[mode], imgs[engine.MODE_FP64]
    l2 = float(np.sqrt(((a - b) ** 2).sum() / max((b ** 2).sum(), 1e-300)))
    return {"image_rel_l2_vs_fp64": l2, "bound": 1e-3, "within_bound": l2 <= 1e-3,
            "same_bb1d_candidates": counts[mode] == counts[engine.MODE_FP64]}


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
    host's cores on a 1-in-S sample of the queries, extrapolated to the full iteration."""
    from oracle import ref
    if not ref.available():
        return {"value": None, "unit": "queries/s", "cores": 0, "kind": "reference",
                "sample": "unavailable: oracle/_ref not built on this machine"}
    cores = os.cpu_count() or 1
    threads = cores
    try:
        with open("/proc/meminfo") as fh:
            avail_gb = int([l for l in fh if l.startswith("MemAvailable")][0].split()[1]) / 1e6
        threads = max(1, min(cores, int((avail_gb - 8) / 5.0)))
    except Exception:
        pass
    ref.set_grid_options(64)
    sess = ref.Session(w, ref.PB2D | ref.BB1D_GRID | ref.PP3D, threads)
    n_seg, n_pt = sess.n_segment, sess.n_point
    total = n_seg + n_pt
    probe_stride = max(1, total // (threads * 8))
    t_probe = sess.eval(1, probe_stride)
    per_query_ms = t_probe / max(1, len(range(1, max(n_seg, n_pt), probe_stride)))
    stride = max(1, int(math.ceil(per_query_ms * max(n_seg, n_pt) / (seconds * 1000.0))))
    t = sess.eval(0, stride)
    sess.close()
    full_ms = sess.build_ms + t * stride
    out = {"value": total / (full_ms / 1000.0), "unit": "queries/s", "cores": threads, "kind": "reference",
           "sample": "reference SmallUPBP estimators (EmbreeBre + PhotonBeamsEvaluator USE_GRID -gridres 64 + "
                     "HashGrid/RangeQuery), one structure set per thread; every %d-th query timed (%.1f s) and "
                     "extrapolated linearly, plus the per-thread build (%.1f s)" % (stride, t / 1000.0,
                                                                                    sess.build_ms / 1000.0),
           "ms_per_iteration": full_ms}
    # the same code on one core: its own build plus a sample about a quarter as long
    one = ref.Session(w, ref.PB2D | ref.BB1D_GRID | ref.PP3D, 1)
    n_max = max(n_seg, n_pt)
    pstride = max(1, n_max // 64)
    per_query1 = one.eval(1, pstride) / max(1, len(range(1, n_max, pstride)))
    stride1 = max(1, int(math.ceil(per_query1 * n_max / (seconds * 250.0))))
    t1 = one.eval(0, stride1)
    one.close()
    ms1 = one.build_ms + t1 * stride1
    out["one_core"] = {"value": total / (ms1 / 1000.0), "unit": "queries/s", "ms_per_iteration": ms1,
                       "sample": "every %d-th query timed on one thread (%.1f s), plus its build (%.1f s)" % (
                           stride1, t1 / 1000.0, one.build_ms / 1000.0)}
    return out


def run_reference(args, cfg, rank, world):
    """--impl reference: the reference's own CPU estimator code on this host's cores."""
    if rank != 0:
        return None
    from oracle import ref
    from smallupbp_b200 import workload as W
    if not ref.available():
        return {"impl": "reference", "unavailable": "oracle/_ref (reference built from its sources) is not present"}
    w = W.make(cfg, iteration=0)
    cores = os.cpu_count() or 1
    threads = cores
    try:
        with open("/proc/meminfo") as fh:
            avail_gb = int([l for l in fh if l.startswith("MemAvailable")][0].split()[1]) / 1e6
        threads = max(1, min(cores, int((avail_gb - 8) / 5.0)))
    except Exception:
        pass
    ref.set_grid_options(64)
    sess = ref.Session(w, ref.PB2D | ref.BB1D_GRID | ref.PP3D, threads)
    n = max(sess.n_segment, sess.n_point)
    total = sess.n_segment + sess.n_point
    probe = sess.eval(1, max(1, n // (threads * 8)))
    per_q = probe / max(1, len(range(1, n, max(1, n // (threads * 8)))))
    stride = max(1, int(math.ceil(per_q * n / (max(1.0, args.cpu_seconds / 2) * 1000.0))))
    for i in range(args.warmup):
        sess.eval(2 + i, stride * 4)
    times = []
    for i in range(args.steps):
        times.append(sess.eval(i % stride, stride))
    sess.close()
    step_ms = sess.build_ms + statistics.mean(times) * stride
    value = total / (step_ms / 1000.0)
    return {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": step_ms, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "impl": "reference",
        "data": "synthetic: seeded UPBP light/camera passes (Philox) in the %s scene; no dataset" % cfg.name,
        "config": dict(workload_desc(cfg), grid_resolution=64),
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": threads, "kind": "reference",
                         "sample": "every %d-th query per step, extrapolated with the per-thread build (%.1f s)" % (
                             stride, sess.build_ms / 1000.0)},
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
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64 (adjoint f64 duals)",
        "data": "synthetic: seeded UPBP light/camera passes (Philox) in the %s scene; no dataset" % cfg.name,
        "config": dict(workload_desc(cfg), mode="mixed forward + dual-number adjoint",
                       loss="sum (I - I_target)^2, target sigma_s=0.7 sigma_a=0.05 g=0.5, at sigma_s=0.5 "
                            "sigma_a=0.1 g=0.3"),
        "adjoint": {"forward_ms": statistics.median(fwd), "backward_ms": statistics.median(bwd),
                    "peak_device_bytes": int(peak), "loss": loss,
                    "grad": {"sigma_a": grads[0], "sigma_s": grads[1], "g": grads[2]}},
    }


def main():
    args = parse()
    rank, world, local_rank = dist_env()
    from smallupbp_b200 import workload as W
    cfg = W.config(args.config)
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

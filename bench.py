#!/usr/bin/env python3
"""Benchmark of the plain volume DMO on the Kuhn tet cube 48^3 (117,649 vertices, 663,552
tetrahedra, 103,823 interior vertices, interior jitter +-0.3h, boundary fixed, mean ratio,
8x8x8 grid, 3 levels, 20 iterations).

One step = one complete 20-iteration optimisation of that mesh from its perturbed state
(positions reset from a device copy at the start of the step; every colour launch of every
iteration plus the per-iteration quality / monotonicity reduction). Metric: vertex updates
per second = interior vertices x 20 x steps / time.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 runs under torchrun: every rank optimises its own copy of the mesh (replicas; the
path has no exchange step), the time is the max over ranks and the value the sum of all
ranks' vertex updates. ``--impl reference`` times the CPU restatement of the reference's
own FP32 kernel (oracle/) on the host cores instead.

The second half of the metric, time-to-plain-DMO min-quality learned vs plain, is the
``learned`` object (rank 0 at N = 1; ``--no-learned`` skips it): the proposal network is
trained from scratch on the GPU on the (ring, DMO displacement) pairs of 20 plain iterations
of a separate seeded 48^3 tet cube; then on the 100^3 tet cube (1,030,301 vertices,
6,000,000 tetrahedra, jitter 0.3h) plain DMO runs 20 iterations, and the learned mode runs
from the same start until its minimum element quality reaches plain's final minimum - 1e-4.
Both times are the sums of per-iteration CUDA-event times.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "vertex-updates/s (plain DMO, tet cube 48^3, 20 iterations)"
UNIT = "vertex-updates/s"
N_ITER = 20
CUBE_N = 48


def workload_config(extra=None):
    cfg = {"workload": "tet cube 48^3 plain DMO (Kuhn, 117649 vertices / 663552 tets, jitter 0.3h, boundary fixed)",
           "mesh_vertices": 117649, "mesh_tets": 663552, "inner_vertices": 103823,
           "iterations_per_step": N_ITER, "grid": "8x8x8", "levels": 3, "quality": "mean ratio",
           "parallelism": "replicas", "l2": "flushed between steps (256 MiB write)"}
    if extra:
        cfg.update(extra)
    return cfg


def rank_info():
    from volumesurfacediscretemeshoptimization_b200 import replicas
    return replicas.rank_info()


class ClockSampler:
    """nvidia-smi clock / throttle samples during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index, period_ms=50):
        self.gpu = gpu_index
        self.period_ms = period_ms
        self.samples = []
        self._p = None
        self._t = None

    def _read(self):
        for line in self._p.stdout:
            line = line.strip()
            if line:
                self.samples.append([x.strip() for x in line.split(",")])

    def __enter__(self):
        try:
            self._p = subprocess.Popen(["nvidia-smi", "-i", str(self.gpu), "--query-gpu=" + self.Q,
                                        "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self._t = threading.Thread(target=self._read, daemon=True)
            self._t.start()
            time.sleep(0.1)   # the first sample before the timed work
        except Exception:
            self._p = None
        return self

    def __exit__(self, *a):
        if self._p is not None:
            time.sleep(self.period_ms / 1e3)
            self._p.terminate()
            try:
                self._p.wait(timeout=5)
            except Exception:
                self._p.kill()
        if self._t:
            self._t.join(timeout=5)

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"], "samples": 0}
        sm = [float(s[1]) for s in self.samples if s[1].replace(".", "").isdigit()]
        mx = [float(s[2]) for s in self.samples if s[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for s in self.samples for i in range(4) if len(s) > 5 + i and s[5 + i] == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.samples)}


_HOST_CPU = None


def host_cpu():
    """(model name, physical cores, logical CPUs usable by this process), read once: after the
    first OpenMP region with OMP_PROC_BIND the main thread is bound to one core, so a later
    sched_getaffinity would report that core alone."""
    global _HOST_CPU
    if _HOST_CPU is None:
        _HOST_CPU = _read_host_cpu()
    return _HOST_CPU


def _read_host_cpu():
    model, cores = None, set()
    try:
        cur = {}
        for line in open("/proc/cpuinfo"):
            if ":" not in line:
                if cur.get("processor") is not None:
                    cores.add((cur.get("physical id", "0"), cur.get("core id", cur["processor"])))
                cur = {}
                continue
            k, v = [x.strip() for x in line.split(":", 1)]
            cur[k] = v
            if k == "model name" and model is None:
                model = v
        if cur.get("processor") is not None:
            cores.add((cur.get("physical id", "0"), cur.get("core id", cur["processor"])))
    except OSError:
        pass
    logical = len(os.sched_getaffinity(0)) if hasattr(os, "sched_getaffinity") else (os.cpu_count() or 1)
    physical = min(len(cores), logical) if cores else logical
    return model, max(1, physical), logical


def pin_openmp(threads):
    """One OpenMP thread per physical core, bound to it; set before the oracle library (and its
    OpenMP runtime) is loaded."""
    os.environ.setdefault("OMP_NUM_THREADS", str(threads))
    os.environ.setdefault("OMP_PLACES", "cores")
    os.environ.setdefault("OMP_PROC_BIND", "close")


def cpu_baseline_sample(xyz, tets, max_seconds=20.0):
    """Times the oracle's literal FP32 restatement of k_optimizeHierarchicalInnerTet on the
    host cores (one pinned OpenMP thread per physical core) over the first colour class(es) of
    the first iteration."""
    model, cores, logical = host_cpu()
    pin_openmp(cores)
    from oracle import oracle as O
    m = O.OracleMesh(O.TET, xyz, tets, color_seed=1)
    x = m.xyz
    done = 0
    t0 = time.perf_counter()
    classes = 0
    for (v0, v1) in m.color_ranges():
        # bound the sample: at most ~max_seconds of CPU work
        if time.perf_counter() - t0 > max_seconds:
            break
        x = m.dmo_color_ref32(x, v0, v1, 0.5, cores)
        done += v1 - v0
        classes += 1
    dt = time.perf_counter() - t0
    return {"value": done / dt, "unit": UNIT, "cores": cores, "kind": "port",
            "cpu_model": model, "logical_cpus": logical,
            "threads": f"{cores} OpenMP threads, OMP_PLACES={os.environ.get('OMP_PLACES')} "
                       f"OMP_PROC_BIND={os.environ.get('OMP_PROC_BIND')}",
            "seconds": dt, "vertex_updates": done,
            "sample": f"first {classes} colour classes ({done} vertex updates) of iteration 1, "
                      f"literal FP32 restatement of the reference kernel (the reference has no CPU DMO), "
                      f"{cores} pinned threads, {dt:.1f} s"}


def reference_gpu_row(xyz, tets):
    """The reference's own CUDA path built from its sources (oracle/_ref/libref_vsdmo.so): its
    mesh build, then its k_optimizeHierarchicalInnerTet<128> over every interior colour for 20
    iterations with its host loop's per-launch synchronisation (the surface passes off: boundary
    fixed), timed with CUDA events. Colouring: its live cusparseScsrcolor, and its own JPL."""
    from oracle import oracle as O
    if O.refvs_lib() is None:
        return {"unavailable": "the reference's CUDA sources were not built into oracle/_ref"}
    out = {"what": "reference kernels on this B200: k_optimizeHierarchicalInnerTet<128>, one block of 128 "
                   "threads per vertex, cudaDeviceSynchronize after each colour launch (dmo/DMOTet.cu:129-136)",
           "workload": "tet cube 48^3, 20 iterations, boundary fixed"}
    for name, mode in (("cusparse_colouring", O.COLOURING_CUSPARSE), ("jpl_colouring", O.COLOURING_JPL)):
        rm = O.RefMesh(O.TET, xyz, tets, colouring=mode)
        n_inner = rm.info["nV"] - rm.info["nSurf"]
        x0 = rm.positions()
        rm.colour_sweeps(3)                    # warm-up
        rm.set_positions(x0)
        ms = rm.colour_sweeps(N_ITER)
        out[name] = {"colours": rm.info["nColorsInner"], "ms": ms,
                     "vertex_updates_per_s": n_inner * N_ITER / (ms / 1e3)}
        rm.close()
    return out


def run_reference(args):
    """The reference arm: each step is one bounded sample (about 8 s) of the CPU restatement of
    the reference kernel on the host cores; value = vertex updates / time over the timed steps.
    The reference's own CUDA path on this GPU is reported beside it (reference_gpu)."""
    r, w, _ = rank_info()
    if r != 0:
        return 0
    from volumesurfacediscretemeshoptimization_b200 import meshgen as G
    xyz, tets = G.config2()
    done = secs = 0.0
    base = None
    for i in range(args.warmup + args.steps):
        b = cpu_baseline_sample(xyz, tets, max_seconds=8.0)
        if i >= args.warmup:
            done += b["vertex_updates"]
            secs += b["seconds"]
            base = b
    v = done / secs
    base["value"] = v
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": UNIT, "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": secs / args.steps * 1e3,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic (seeded Kuhn tet cube; the reference ships no meshes)",
            "config": workload_config({"step": "one bounded CPU sample of the workload (see cpu_baseline)"}),
            "cpu_baseline": base,
            "e2e": {"value": v, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    if not args.no_reference_gpu:
        try:
            line["reference_gpu"] = reference_gpu_row(xyz, tets)
        except Exception as e:  # a checker row: its absence must not lose the reference line
            line["reference_gpu"] = {"unavailable": f"{type(e).__name__}: {e}"}
    print(json.dumps(line), flush=True)
    return 0


def run_ours(args):
    import torch
    from volumesurfacediscretemeshoptimization_b200 import replicas
    r, world, lr = rank_info()
    dist = replicas.init("nccl", timeout_s=120)
    torch.cuda.set_device(lr)
    dev = torch.device("cuda", lr)
    from volumesurfacediscretemeshoptimization_b200 import build as B
    if not os.path.exists(B.LIB_PATH):
        raise SystemExit("libvsdmo.so missing: run __graft_entry__.build() first")
    import volumesurfacediscretemeshoptimization_b200 as V
    from volumesurfacediscretemeshoptimization_b200 import meshgen as G, _capi

    lib = _capi.lib()
    stream = torch.cuda.Stream(device=dev)
    sp = stream.cuda_stream
    xyz, tets = G.config2(seed=replicas.replica_seed(r))
    # ---- device-resident workload -------------------------------------------------------------
    mesh = V._Mesh.__new__(V.DMOMeshTet)
    with torch.cuda.stream(stream):
        d_xyz = torch.from_numpy(xyz).to(dev)
        d_tets = torch.from_numpy(tets).to(dev)
        stream.synchronize()
        V.DMOMeshTet.__init__(mesh, None, None, 1, sp, (d_xyz.data_ptr(), d_tets.data_ptr(), len(xyz), len(tets)))
    n_inner = mesh.info["nV"] - mesh.info["nSurf"]
    opt = V.DMOTetClass(mesh, n_iter=10 ** 9)
    launches_per_iter = opt.launches_per_iteration   # colour launches + the quality kernel
    x0 = torch.empty(len(xyz) * 3, dtype=torch.float32, device=dev)
    mesh.positions_to_device(x0.data_ptr(), original_order=False)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def reset():
        _capi.check(lib.vsdmo_mesh_set_positions(mesh.h, C.c_void_p(x0.data_ptr()), 0, _capi.DEVICE))

    def step():
        reset()
        opt.restart()
        opt.iterate(N_ITER)

    for _ in range(max(args.warmup, 0)):
        step()
    torch.cuda.synchronize()
    q_final = opt.getQuality()
    # ---- timed region ----------------------------------------------------------------------------
    # events around every step and around every iteration inside it (one graph replay: the colour
    # launches of k_dmo_tet and the quality reduction)
    ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    it_ev = [[torch.cuda.Event(enable_timing=True) for _ in range(N_ITER + 1)] for _ in range(args.steps)]
    replicas.barrier(dist)
    torch.cuda.synchronize()
    with ClockSampler(lr) as clk:
        for i in range(args.steps):
            with torch.cuda.stream(stream):
                flush.fill_(float(i))
                ev[i][0].record(stream)
                reset()
                opt.restart()
                it_ev[i][0].record(stream)
                for k in range(N_ITER):
                    opt.iterate(1)
                    it_ev[i][k + 1].record(stream)
                ev[i][1].record(stream)
        torch.cuda.synchronize()
    replicas.barrier(dist)
    ms = sum(a.elapsed_time(b) for a, b in ev)
    ms_max = replicas.max_over_ranks(ms, dist, dev)
    value = replicas.whole_job_rate(n_inner * N_ITER * args.steps, ms_max, world)
    iter_ms = sum(it_ev[i][0].elapsed_time(it_ev[i][N_ITER]) for i in range(args.steps)) / args.steps
    clocks = clk.summary()

    # ---- roofline of the grid-search kernel, inside the timed steps ------------------------------------
    n_col = mesh.info["nColorsInner"]
    peaks = {}
    try:
        peaks = json.load(open(os.path.join(ROOT, "MEASURED_PEAKS.json")))
    except Exception:
        pass
    prof = {}
    try:
        prof = json.load(open(os.path.join(ROOT, "profiles", "dmo_tet_config2_traffic.json")))
    except Exception:
        pass
    # k_dmo_tet's share of an iteration's device time (one launch per colour class + the quality
    # reduction), from the ncu launch list of profile_cases.py tet (profiles/k_dmo_tet_config2.md)
    share = prof.get("share_of_iteration", 0.988)
    kern_ms_step = iter_ms * share
    launches_step = n_col * N_ITER
    avg_launch_s = kern_ms_step / launches_step / 1e3
    upd_per_launch = n_inner / n_col
    sm_mhz = clocks.get("sm_mhz") or 1965.0
    inst_per_update = prof.get("warp_instructions_per_vertex_update")
    bytes_per_update = 488  # 20 + 12k + 12|N| + 12 with k = 24 tets and |N| = 14 neighbours (interior Kuhn vertex)
    hbm_peak = peaks.get("hbm_gbs") or 6650.0
    hbm_achieved = bytes_per_update * upd_per_launch / avg_launch_s / 1e9
    issue_peak = 148 * 4 * sm_mhz * 1e6  # warp instructions per second: 4 schedulers x 148 SMs x clock
    issue_achieved = inst_per_update * upd_per_launch / avg_launch_s if inst_per_update else None
    traffic = prof.get("dram_bytes_per_vertex_update")
    roofline = {
        "bound": "issue", "kernel": "k_dmo_tet",
        "achieved": issue_achieved, "peak": issue_peak, "unit": "warp-instructions/s",
        "frac": issue_achieved / issue_peak if issue_achieved else None,
        "traffic": traffic * upd_per_launch if traffic else None,
        "per": "one launch (one colour class, average over the timed steps)",
        "how": "achieved = warp instructions per vertex update (ncu smsp__inst_executed.sum on this workload, "
               "profiles/k_dmo_tet_config2.md) x vertex updates per launch / average launch time; peak = 148 SMs "
               "x 4 schedulers x median SM clock during the timed region; launch time = per-iteration CUDA "
               "events inside the timed steps x k_dmo_tet's share of an iteration (ncu launch list)",
        "warp_instructions_per_vertex_update": inst_per_update,
        "kernel_ms_per_step": kern_ms_step, "iteration_ms_per_step": iter_ms,
        "share_of_iteration": share, "launches_per_step": launches_step,
        "hbm": {"achieved": hbm_achieved, "peak": hbm_peak, "unit": "GB/s", "frac": hbm_achieved / hbm_peak,
                "peak_source": "measured" if peaks.get("hbm_gbs") else "fallback",
                "algorithmic_bytes_per_vertex_update": bytes_per_update,
                "dram_bytes_per_vertex_update": traffic,
                "traffic_over_algorithmic": traffic / bytes_per_update if traffic else None},
    }
    assert kern_ms_step <= ms_max / args.steps * 1.0001 or world > 1

    # ---- end to end through the public API with host buffers ---------------------------------------------
    pin_xyz = torch.from_numpy(xyz).pin_memory()
    pin_tets = torch.from_numpy(tets).pin_memory()
    out_host = torch.empty(len(xyz) * 3, dtype=torch.float32).pin_memory()
    e2e_ms = []
    for i in range(max(1, min(args.steps, 3)) + 1):
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        with torch.cuda.stream(stream):
            a.record(stream)
            m2 = V._Mesh.__new__(V.DMOMeshTet)
            h = C.c_void_p()
            _capi.check(lib.vsdmo_mesh_create(_capi.TET, C.c_void_p(pin_xyz.data_ptr()), len(xyz),
                                              C.c_void_p(pin_tets.data_ptr()), len(tets), _capi.HOST, 1,
                                              C.c_void_p(sp), C.byref(h)))
            m2.h = h
            m2.info = {n: lib.vsdmo_mesh_info(h, j) for j, n in enumerate(V.INFO_NAMES)}
            m2.nVertices = m2.info["nV"]
            o2 = V.DMOTetClass(m2, n_iter=N_ITER)
            o2.optimize()
            _capi.check(lib.vsdmo_mesh_get_positions(h, C.c_void_p(out_host.data_ptr()), 1, _capi.HOST))
            b.record(stream)
        torch.cuda.synchronize()
        o2.close()
        m2.close()
        if i > 0:  # first one is a warm-up
            e2e_ms.append(a.elapsed_time(b))
    e2e_ms_med = replicas.max_over_ranks(statistics.median(e2e_ms), dist, dev)
    e2e_value = replicas.whole_job_rate(n_inner * N_ITER, e2e_ms_med, world)

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_max / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic (seeded Kuhn tet cube; the reference ships no meshes)",
        "config": workload_config({"final_min_quality": q_final, "colours": n_col}),
        "clocks": clocks,
        "gpu_launches": (launches_per_iter * N_ITER + 2) * args.steps,
        "e2e": {"value": e2e_value, "unit": UNIT, "ms_per_step": e2e_ms_med,
                "h2d_bytes_per_step": int(xyz.nbytes + tets.nbytes), "d2h_bytes_per_step": int(xyz.nbytes),
                "includes": "mesh build (connectivity + colouring) from pinned host arrays, 20 iterations, positions back to host"},
        "roofline": roofline,
    }
    opt.close()
    mesh.close()
    if r == 0 and world == 1 and not args.no_colour_priority:
        line["colour_priority"] = colour_priority_rates(dev, stream, xyz, tets, value, n_col, q_final)
    if r == 0 and world == 1 and not args.no_learned:
        line["learned"] = learned_time_to_quality(dev, stream)
    if r == 0 and world == 1 and not args.no_batched:
        line["batched"] = batched_throughput(dev, stream)
    if r == 0 and world == 1 and not args.no_surface:
        line["surface"] = surface_rates(dev, stream)
    if r == 0 and world == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline_sample(xyz, tets)
    # compact summaries last, where a tail of the line still shows them
    summary = {"vertex_updates_per_s": value, "e2e_vertex_updates_per_s": e2e_value,
               "issue_frac": roofline["frac"], "hbm_frac": roofline["hbm"]["frac"]}
    if "learned" in line:
        L = line["learned"]
        summary["learned"] = {"time_ratio_learned_over_plain": L["time_ratio_learned_over_plain"],
                              "held_out_ratio": L["held_out"]["time_ratio_learned_over_plain"],
                              "learned_reached": L["learned_reached"], "learned_iterations": L["learned_iterations"],
                              "plain_ms": L["plain_ms"], "learned_ms": L["learned_ms"],
                              "excludes": "training (" + str(L["training"].get("train_s")) + " s) and pair "
                                          "collection: one-off, on a separate 48^3 mesh"}
    if "batched" in line:
        B = line["batched"]
        summary["batched"] = {"reference_config_vertex_updates_per_s": B["reference_config"]["vertex_updates_per_s"],
                              "autotuned_vertex_updates_per_s": B["autotuned"]["vertex_updates_per_s"],
                              "per_mesh_loop_vertex_updates_per_s": B["per_mesh_loop"]["vertex_updates_per_s"]}
    if "colour_priority" in line:
        summary["colour_priority"] = {k: line["colour_priority"][k]["vertex_updates_per_s"]
                                      for k in ("default", "hash_rounds", "reference")}
    if "surface" in line:
        summary["surface_vertex_updates_per_s"] = {k: v["vertex_updates_per_s"] for k, v in line["surface"].items()
                                                   if isinstance(v, dict)}
    line["summary"] = summary
    if r == 0:
        print(json.dumps(line), flush=True)
    replicas.finish(dist)
    return 0


def colour_priority_rates(dev, stream, xyz, tets, hash_value, hash_colours, hash_min_q):
    """The same 20-iteration plain DMO under the other colourings: round colours (the
    reference's rule) with the default hashed priorities (COLOR_ROUNDS | 1), and with the
    reference's own priorities n - i (COLOR_REFERENCE); one warm-up and one timed run each."""
    import torch
    import volumesurfacediscretemeshoptimization_b200 as V
    sp = stream.cuda_stream
    out = {"default": {"colours": hash_colours, "vertex_updates_per_s": hash_value, "final_min_quality": hash_min_q}}
    for name, seed in (("hash_rounds", V.COLOR_ROUNDS | 1), ("reference", V.COLOR_REFERENCE)):
        m = V.DMOMeshTet(xyz, tets, color_seed=seed, stream=sp)
        n_inner = m.info["nV"] - m.info["nSurf"]
        o = V.DMOTetClass(m, n_iter=10 ** 9)
        x0 = m.positions()
        o.iterate(3)
        m.set_positions(x0)
        o.restart()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
            o.iterate(N_ITER)
            b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        out[name] = {"colours": m.info["nColorsInner"], "vertex_updates_per_s": n_inner * N_ITER / (ms / 1e3),
                     "ms": ms, "final_min_quality": o.getQuality()}
        o.close()
        m.close()
    out["how"] = ("default = the seeded hash priorities, each vertex taking the smallest colour its higher-priority "
                  "neighbours leave free; hash_rounds = the same priorities, colour = JPL round (the reference's rule, "
                  "mesh/VertexColoring.cu:76-105); reference = round colours with the reference's priorities n - i "
                  "(mesh/VertexColoring.cu:107-125); same mesh, 20 iterations, no L2 flush")
    return out


ONCE_AFTER = 1   # first iteration of the one-launch-per-iteration proposal schedule (variant)


def learned_time_to_quality(dev, stream):
    """Trains the proposal network on plain-DMO pairs, then times plain vs learned DMO on the
    100^3 tet cube to plain's final (20-iteration) minimum quality."""
    import torch
    import volumesurfacediscretemeshoptimization_b200 as V
    from volumesurfacediscretemeshoptimization_b200 import meshgen as G
    from volumesurfacediscretemeshoptimization_b200.learned import DEFAULTS as LEARNED_CFG, train_proposal
    sp = stream.cuda_stream
    model, training = train_proposal(stream, LEARNED_CFG)
    # evaluation mesh
    xyz5, tets5 = G.config5()
    m5 = V.DMOMeshTet(xyz5, tets5, stream=sp)
    n5 = m5.info["nV"] - m5.info["nSurf"]
    x0 = m5.positions()

    def measure(once_after):
        o5 = V.DMOTetClass(m5, n_iter=10 ** 9)

        def run(stop_q, max_it):
            ts, qs = [], []
            for _ in range(max_it):
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                with torch.cuda.stream(stream):
                    a.record(stream)
                    o5.iterate(1)
                    b.record(stream)
                torch.cuda.synchronize()
                ts.append(a.elapsed_time(b))
                qs.append(o5.getQuality())
                if stop_q is not None and qs[-1] >= stop_q:
                    break
            return ts, qs

        m5.set_positions(x0); o5.restart()
        run(None, 3)                                   # warm-up (graph capture, clocks)
        m5.set_positions(x0); o5.restart()
        tp, qp = run(None, N_ITER)
        target = qp[-1] - 1e-4
        m5.set_positions(x0); o5.restart()
        o5.set_model(model, LEARNED_CFG["reduced_n"], LEARNED_CFG["reduced_depth"], LEARNED_CFG["reduced_scale"])
        o5.set_proposal_schedule(once_after)
        run(None, max(2, once_after + 2))              # warm-up of the learned graph(s)
        m5.set_positions(x0); o5.restart()
        tl, ql = run(target, 4 * N_ITER)
        counters = o5.learned_counters()
        o5.close()
        return tp, qp, target, tl, ql, counters

    tp, qp, target, tl, ql, (acc, fb, fb_moved, _) = measure(-1)
    reached = ql[-1] >= target
    tpa, qpa, targeta, tla, qla, (acca, fba, _, _) = measure(ONCE_AFTER)
    reacheda = qla[-1] >= targeta
    m5.close()
    # the same model and settings on the cube jittered with another seed (not used to choose them)
    xyz5, tets5 = G.config5(seed=2)
    m5 = V.DMOMeshTet(xyz5, tets5, stream=sp)
    x0 = m5.positions()
    tph, qph, targeth, tlh, qlh, _ = measure(-1)
    reachedh = qlh[-1] >= targeth
    m5.close(); model.close()
    return {
        "workload": "tet cube 100^3 (1030301 vertices / 6000000 tets, jitter 0.3h, boundary fixed), seed 0",
        "plain_ms": sum(tp), "plain_iterations": len(tp), "plain_final_min_quality": qp[-1],
        "target_min_quality": target,
        "learned_ms": sum(tl) if reached else None, "learned_iterations": len(tl), "learned_reached": bool(reached),
        "learned_final_min_quality": ql[-1],
        "time_ratio_learned_over_plain": (sum(tl) / sum(tp)) if reached else None,
        "plain_vertex_updates_per_s": n5 * len(tp) / (sum(tp) / 1e3),
        "reduced_accepted": acc, "fallbacks": fb, "fallbacks_moved": fb_moved,
        "reduced_accept_fraction": acc / max(1, acc + fb),
        "search": {k: LEARNED_CFG[k] for k in ("reduced_n", "reduced_depth", "reduced_scale")},
        "training": training,
        "plain_ms_per_iteration": tp, "learned_ms_per_iteration": tl,
        "proposals_once_per_iteration": {
            "how": f"from iteration {ONCE_AFTER} on the network runs once per iteration for all interior "
                   "vertices (positions at the iteration's start) instead of before every colour class; "
                   "plain arm rerun",
            "plain_ms": sum(tpa), "plain_final_min_quality": qpa[-1], "target_min_quality": targeta,
            "learned_ms": sum(tla) if reacheda else None, "learned_iterations": len(tla),
            "learned_reached": bool(reacheda),
            "time_ratio_learned_over_plain": (sum(tla) / sum(tpa)) if reacheda else None,
            "reduced_accepted": acca, "fallbacks": fba,
            "plain_ms_per_iteration": tpa, "learned_ms_per_iteration": tla},
        "held_out": {"workload": "tet cube 100^3, jitter 0.3h, seed 2", "plain_ms": sum(tph),
                     "plain_final_min_quality": qph[-1], "learned_ms": sum(tlh) if reachedh else None,
                     "learned_iterations": len(tlh), "learned_reached": bool(reachedh),
                     "time_ratio_learned_over_plain": (sum(tlh) / sum(tph)) if reachedh else None},
        "timing": "sum of per-iteration CUDA-event times on the library stream",
    }


BATCH_ITERS = 10
SURF_ITERS = 15


def surface_rates(dev, stream):
    """The surface workloads with their feature passes on: the level-7 icosphere (triangles,
    DMOTriClass) and the 512 x 256 torus (quads, DMOQuadClass), tangential noise 0.35 of the
    local edge length and normal noise N(0, 1e-3), 15 iterations. One warm-up iteration (graph
    capture), positions reset, then the 15 timed iterations (CUDA events on the library stream).
    A vertex update is one vertex moved by its pass: every surface vertex is visited once per
    iteration, free vertices by the surface search and feature vertices by the curve search."""
    import torch
    import volumesurfacediscretemeshoptimization_b200 as V
    from volumesurfacediscretemeshoptimization_b200 import meshgen as G
    sp = stream.cuda_stream
    out = {}
    for name, gen, mcls, ocls in (("config3_tri", G.config3_tri, V.DMOMeshTri, V.DMOTriClass),
                                  ("config3_quad", G.config3_quad, V.DMOMeshQuad, V.DMOQuadClass)):
        xyz, el = gen()
        m = mcls(xyz, el, stream=sp)
        o = ocls(m, n_iter=SURF_ITERS)
        o.iterate(1)
        m.set_positions(xyz, original_order=True)
        o.restart()
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
            o.iterate(SURF_ITERS)
            b.record(stream)
        torch.cuda.synchronize()
        ms = a.elapsed_time(b)
        mn, mean = o.quality_stats()
        n_upd = m.info["nSurf"]
        out[name] = {"vertices": m.info["nV"], "feature_vertices": m.info["nFeature"], "iterations": SURF_ITERS,
                     "ms": ms, "vertex_updates_per_s": n_upd * SURF_ITERS / (ms / 1e3),
                     "final_min_quality": mn, "final_mean_quality": mean,
                     "launches_per_iteration": o.launches_per_iteration}
        o.close()
        m.close()
    out["workload"] = ("icosphere level 7 (163842 vertices) and torus 512x256 quads (131072 vertices), tangential "
                       "noise 0.35 local edge, normal N(0, 1e-3), seed 0, feature vertices sliding on their curves")
    return out


def batched_throughput(dev, stream):
    """256 flat tri / quad meshes (vertex counts log-uniform in [500, 50,000], jitter 0.4h)
    optimised together: one persistent launch per iteration replayed from a CUDA graph, with
    the reference configuration (8 per axis, 3 levels, one warp per vertex) and with the
    autotuned per-bucket configuration, against a loop over one single-mesh optimiser per mesh
    (the reference runs one mesh per DMOTriFlatClass object). 10 iterations each, from the
    same start; CUDA-event times on the library stream."""
    import torch
    import volumesurfacediscretemeshoptimization_b200 as V
    from volumesurfacediscretemeshoptimization_b200 import meshgen as G
    sp = stream.cuda_stream
    meshes = G.config4()
    t0 = time.perf_counter()
    b = V.BatchDMO(meshes, stream=sp)
    build_s = time.perf_counter() - t0
    x0 = b.positions()
    infos = [b.mesh_info(i) for i in range(len(meshes))]
    n_free = sum(m["free_end"] - m["free_begin"] for m in infos)

    def timed(n):
        a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        with torch.cuda.stream(stream):
            a.record(stream)
            b.iterate_async(n)
            e.record(stream)
        b.sync()
        torch.cuda.synchronize()
        return a.elapsed_time(e)

    def summary():
        mn, mean, _ = b.stats(BATCH_ITERS)
        return {"min_of_min_quality": float(mn.min()), "mean_of_mean_quality": float(mean.mean())}

    def run_config():
        timed(2)                                  # warm-up (graph capture, clocks)
        b.set_positions(x0); b.restart()
        ms = timed(BATCH_ITERS)
        return ms, summary()

    ms_ref, q_ref = run_config()
    t1 = time.perf_counter()
    report = b.autotune(probe_iters=3)
    tune_s = time.perf_counter() - t1
    b.set_positions(x0); b.restart()
    ms_tuned, q_tuned = run_config()
    info = b.info()
    nq, depth, lanes = b.config()
    b.close()
    # the per-mesh loop: one single-mesh optimiser per mesh, each iterated in turn
    objs = []
    for t, xyz, el in meshes:
        m = (V.DMOMeshTri if t == 0 else V.DMOMeshQuad)(xyz, el, stream=sp)
        o = (V.DMOTriFlatClass if t == 0 else V.DMOQuadFlatClass)(m, n_iter=BATCH_ITERS)
        o.iterate(1)                              # warm-up (graph capture)
        m.set_positions(xyz, original_order=True)
        o.restart()
        objs.append((m, o))
    torch.cuda.synchronize()
    a, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    with torch.cuda.stream(stream):
        a.record(stream)
        for m, o in objs:
            o.iterate(BATCH_ITERS)
        e.record(stream)
    torch.cuda.synchronize()
    ms_loop = a.elapsed_time(e)
    for m, o in objs:
        o.close(); m.close()
    ups = lambda ms: n_free * BATCH_ITERS / (ms / 1e3)
    return {
        "workload": "256 flat grids, tri and quad alternating, vertices log-uniform in [500, 50000] "
                    "(3261948 vertices), jitter 0.4h, boundary fixed, seed 0",
        "free_vertices": n_free, "iterations": BATCH_ITERS,
        "reference_config": {"ms": ms_ref, "vertex_updates_per_s": ups(ms_ref), **q_ref,
                             "grid": "8x8", "levels": 3, "lanes_per_vertex": 32},
        "autotuned": {"ms": ms_tuned, "vertex_updates_per_s": ups(ms_tuned), **q_tuned,
                      "buckets": report.strip().splitlines(), "autotune_s": tune_s,
                      "configs_used": sorted({(int(a), int(b_), int(c)) for a, b_, c in zip(nq, depth, lanes)})},
        "per_mesh_loop": {"ms": ms_loop, "vertex_updates_per_s": ups(ms_loop),
                          "how": "256 single-mesh optimisers (8x8, 3 levels), each iterate(10) in turn"},
        "speedup_batched_over_loop": ms_loop / ms_ref,
        "work_items_per_iteration": info["items"], "colour_classes": info["colors"],
        "persistent_ctas": info["blocks"], "build_s": build_s,
        "timing": "CUDA events on the library stream; one graph replay per iteration",
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-learned", action="store_true")
    ap.add_argument("--no-batched", action="store_true")
    ap.add_argument("--no-reference-gpu", action="store_true")
    ap.add_argument("--no-colour-priority", action="store_true")
    ap.add_argument("--no-surface", action="store_true")
    args = ap.parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

#!/usr/bin/env python3
"""Benchmark of the B200 corotational elastic solve (PCG DOF-iterations per second).

One step = one fixed step of the 64^3 mixed-material block (262,144 REVs,
wood/iron/stone/aluminium, bottom layer fixed, gravity -9.81, dt 1 ms): the
rotation fit, 5 corotational passes (assembly + FP32 inner block-Jacobi PCG
inside FP64 iterative refinement to a true relative residual of 1e-8, the
rotation re-fit between passes) and the bond-stress evaluation. Every step
starts from the same resident state (device-side checkpoint restore).

  python bench.py [--gpus N --steps K --warmup W] [--impl reference]

With --gpus N > 1 it runs under torchrun with one rank per GPU; every rank
solves its own scene (weak scaling, no data-path collective) and the device
time is the max over ranks. --impl reference times the reference's own CPU
block-Jacobi PCG loop (restated f32 port, all host threads) on the same
system and prints the same JSON line with "impl": "reference".
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time
from pathlib import Path

ROOT = Path(__file__).resolve().parent
sys.path[:0] = [str(ROOT / "voxel-sim_b200"), str(ROOT / "oracle")]

import numpy as np  # noqa: E402

BYTES_PER_REV = {  # canonical algorithmic bytes per active REV and PCG iteration
    "matvec_f32": 136, "update_f32": 108, "direction_f32": 36,
    "matvec_f64": 256, "update_f64": 216, "direction_f64": 72,
}
METRIC = "PCG DOF-iters/s (FP32 inner PCG in FP64 refinement to 1e-8)"


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mixed_block",
                    choices=["mixed_block", "wood_cube", "damaged_lattice", "batched", "served", "contact"])
    ap.add_argument("--rate", type=float, default=200.0, help="served: Poisson arrivals per second")
    ap.add_argument("--window", type=float, default=5.0, help="served: seconds of arrivals")
    ap.add_argument("--drain", type=float, default=60.0, help="served: seconds to wait for completions")
    ap.add_argument("--request-steps", type=int, default=100, help="served: fixed steps per request")
    ap.add_argument("--slots", type=int, default=256, help="served: resident scenes at most")
    ap.add_argument("--lanes", type=int, default=3, help="served: pools by scene size, each with its own stream")
    ap.add_argument("--no-fp64-compare", action="store_true",
                    help="served: skip the plain FP64 single-scene solves of the template scenes")
    ap.add_argument("--scenes", type=int, default=512, help="batched: scenes per batch")
    ap.add_argument("--pool-kernel", default="auto", choices=["auto", "persistent", "streaming"],
                    help="batched: inner solves in tile kernels (auto, streaming) or persistent waves")
    ap.add_argument("--fp64-sample", type=int, default=None,
                    help="batched: scenes timed in the plain FP64 single-scene form (default all)")
    ap.add_argument("--edge", type=int, default=None)
    ap.add_argument("--passes", type=int, default=None)
    ap.add_argument("--tolerance", type=float, default=None,
                    help="pass target (default: the workload's, 1e-8; 1e-10 for the wood cube)")
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"],
                    help="the FP32-inner / FP64-refinement form, or the plain FP64 form")
    ap.add_argument("--inner-tolerance", type=float, default=0.0,
                    help="relative tolerance of each FP32 inner solve (0 = the library's default)")
    ap.add_argument("--max-iterations", type=int, default=50000)
    ap.add_argument("--cpu-iterations", type=int, default=400, help="PCG iterations per CPU sample")
    ap.add_argument("--cpu-seconds", type=float, default=10.0,
                    help="cpu_baseline: repeat CPU samples until this much time has passed")
    ap.add_argument("--no-oracle-error", action="store_true",
                    help="skip the C oracle's FP64 solve that the mixed pass is compared with")
    ap.add_argument("--no-batched-ratio", action="store_true",
                    help="skip the batched-vs-FP64 single-scene comparison in the default line")
    ap.add_argument("--batched-ratio-scenes", type=int, default=64,
                    help="scenes in the default line's batched comparison")
    ap.add_argument("--no-large-matvec", action="store_true",
                    help="skip the streaming matvec timing on the 160^3 damaged lattice")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    a = ap.parse_args()
    if a.tolerance is None:
        a.tolerance = 1e-10 if a.workload == "wood_cube" else 1e-8
    return a


def build_workload(name, edge, seed):
    from vxsim import scenes as S
    if name == "mixed_block":
        return S.mixed_block(edge or 64, seed=seed)
    if name == "wood_cube":
        return S.wood_cube(edge or 10)
    return S.damaged_lattice(edge or 160, seed=seed)


def predicted_positions(scene, h, gravity):
    """Explicit prediction of src/solver.rs:500-523 from rest (v0 = 0)."""
    from vxsim import scenes as S
    return S.predict_from_rest(scene, h, gravity)


def workload_config(args, scene, world):
    """The `config` of a workload's line, the same in both arms."""
    meta = scene.meta
    return {"workload": f"{meta['workload']} {meta.get('edge')}^3", "revs": scene.n,
            "dof_nominal": 3 * scene.n, "dof_active": int(scene.free_mask().sum()),
            "passes": args.passes or meta["passes"], "tolerance": args.tolerance,
            "precision": "plain FP64 PCG" if args.precision == "fp64" else "FP32 inner PCG, FP64 refinement",
            "l2": "256 MiB buffer written between timed steps", "parallelism": f"replicas{world}"}


def persistent_kernel_name(form, tuning):
    """The on-chip kernel the scene's inner solve runs: its plan and, for the
    range plan, the block size the autotuner chose (VX_PERSIST_RANGE_*)."""
    from vxsim import native as N
    if form == "brick":
        return "k_pcg_brick"
    if form == "expanded":
        return "k_pcg_expanded, 512 threads/block"
    threads = 512
    if tuning and tuning.get("kernel") == N.KERNEL_PERSISTENT:
        threads = N.RANGE_THREADS.get(tuning["blocks_per_sm"], 512)
    return f"k_pcg_persistent, {threads} threads/block"


def measured_peak():
    p = ROOT / "MEASURED_PEAKS.json"
    if p.exists():
        d = json.loads(p.read_text())
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def profiled_traffic():
    p = ROOT / "profiles" / "roofline_traffic.json"
    if p.exists():
        try:
            return json.loads(p.read_text())
        except Exception:
            return None
    return None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        rows = []
        for line in Path(self.path).read_text().splitlines():
            parts = [x.strip() for x in line.split(",")]
            if len(parts) >= 9:
                rows.append(parts)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[k] for r in rows for k in range(4) if r[5 + k].lower() == "active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def cpu_reference_rate(scene, h, pred, iterations, threads, min_seconds):
    """The reference's CPU block-Jacobi PCG loop (f32 port) on pass 0 of the scene:
    samples of `iterations` iterations repeated until `min_seconds` have passed."""
    import pyoracle as O
    o = O.OracleScene(scene)
    o.fit_rotations()
    o.assemble(h, pred)
    rows = o.pack_rows()
    dof = 3 * rows["n"]
    O.pcg_rows_f32(rows, max(2, iterations // 8), 0.0, threads)  # warm the pages and threads
    it, dt, samples = 0, 0.0, 0
    while samples == 0 or dt < min_seconds:
        t0 = time.perf_counter()
        _, k, _ = O.pcg_rows_f32(rows, iterations, 0.0, threads)
        dt += time.perf_counter() - t0
        it += k
        samples += 1
    return rows, dof, it, dt, samples


def large_matvec(ctx, flush, peak, edge=160):
    """The streaming FP32 matvec on the damaged lattice of `edge`^3 REVs (inputs
    well above L2), launched alone after an L2 flush, CUDA events on the scene's
    stream: its fraction of measured HBM against the canonical 136 B per REV."""
    from vxsim import native as N
    from vxsim import scenes as S
    s = S.damaged_lattice(edge, seed=2)
    d = N.DeviceScene(ctx, s)
    d.set_predicted(s.position)
    d.fit_rotations()
    d.corotational_pass(1e-3, 1e-8, 1, precision=N.PRECISION_MIXED, kernel=N.KERNEL_STREAMING)
    t = d.kernel_times(N.PRECISION_MIXED, reps=20, flush_ptr=flush.data_ptr(), flush_bytes=flush.numel())
    active = s.active_count()
    d.close()
    gbs = BYTES_PER_REV["matvec_f32"] * active / (t["matvec_us"] * 1e-6) / 1e9
    return {"workload": f"damaged_lattice {edge}^3", "active_revs": active, "matvec_us_cold_l2": t["matvec_us"],
            "update_us_cold_l2": t["update_us"], "matvec_gbs": gbs, "frac": gbs / peak,
            "bytes_per_rev": BYTES_PER_REV["matvec_f32"]}


def oracle_first_pass(scene, h, pred, tolerance):
    """The C oracle's first pass of the step in FP64 (rotation fit, assembly on
    the prediction, block-Jacobi PCG to `tolerance`): the checker that the
    mixed pass's displacement is compared with."""
    import pyoracle as O
    o = O.OracleScene(scene)
    o.fit_rotations()
    t0 = time.perf_counter()
    it, res = o.solve_coupled(h, 200000, tolerance, predicted=pred)
    return o.positions() - scene.position, it, res, time.perf_counter() - t0


def reference_arm(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    import pyoracle as O
    scene = build_workload(args.workload, args.edge, seed=1)
    meta = scene.meta
    h = meta["dt"] / meta["substeps"]
    pred = predicted_positions(scene, h, meta["gravity"])
    threads = os.cpu_count() or 1
    o = O.OracleScene(scene)
    o.fit_rotations()
    o.assemble(h, pred)
    rows = o.pack_rows()
    dof = 3 * rows["n"]
    for _ in range(args.warmup):
        O.pcg_rows_f32(rows, max(2, args.cpu_iterations // 4), 0.0, threads)
    total_it, total_s = 0, 0.0
    for _ in range(args.steps):
        t0 = time.perf_counter()
        _, it, _ = O.pcg_rows_f32(rows, args.cpu_iterations, 0.0, threads)
        total_s += time.perf_counter() - t0
        total_it += it
    value = dof * total_it / total_s
    sample = (f"{args.cpu_iterations} iterations per step of the reference's CPU block-Jacobi PCG loop "
              f"(src/solver.rs:1833-1911, restated in C, f32 vectors, f64 dots) on pass 0 of {meta['workload']} "
              f"{meta.get('edge')}^3 ({rows['n']} active REVs)")
    line = {
        "impl": "reference", "metric": "PCG DOF-iters/s (plain FP64 PCG)" if args.precision == "fp64" else METRIC,
        "value": value, "unit": "DOF-iter/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000 * total_s / args.steps,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(args, scene, args.gpus),
        "cpu_baseline": {"value": value, "unit": "DOF-iter/s", "cores": threads, "kind": "port", "sample": sample,
                         "omp_num_threads": threads, "host_cpus": os.cpu_count()},
        "e2e": {"value": value, "unit": "DOF-iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def combine_ranks(ms, dof_iters, solves, dist=None, device="cpu"):
    """Whole-job figures of the replica run: the device time is the maximum over
    ranks (every rank's timed region ends at a barrier), the work the sum. Each
    rank takes the same two collectives in the same order."""
    if dist is None:
        return ms, dof_iters, solves
    import torch
    t = torch.tensor([ms], device=device, dtype=torch.float64)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    w = torch.tensor([dof_iters, solves], device=device, dtype=torch.float64)
    dist.all_reduce(w, op=dist.ReduceOp.SUM)
    return float(t.item()), float(w[0].item()), float(w[1].item())


def our_arm(args):
    import torch
    from vxsim import native as N

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    torch.cuda.set_device(local)

    scene = build_workload(args.workload, args.edge, seed=1 + rank)
    meta = scene.meta
    passes = args.passes or meta["passes"]
    h = meta["dt"] / meta["substeps"]
    pred = predicted_positions(scene, h, meta["gravity"])
    free_dof = int(scene.free_mask().sum())
    active = scene.active_count()
    precision = N.PRECISION_FP64 if args.precision == "fp64" else N.PRECISION_MIXED

    ctx = N.Context(local)
    ds = N.DeviceScene(ctx, scene)
    ds.set_predicted(pred)
    ds.save_state()
    ext = torch.cuda.ExternalStream(ds.stream_ptr, device=torch.device("cuda", local))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def step(fetch=False):
        ds.restore_state()
        ds.fit_rotations()
        it = 0
        launches = 1
        worst = 0.0
        for p in range(passes):
            st = ds.corotational_pass(h, args.tolerance, args.max_iterations, precision=precision,
                                      inner_tolerance=args.inner_tolerance)
            it += st["iterations"]
            launches += st["kernel_launches"]
            worst = max(worst, st["true_residual"])
            if p + 1 < passes:
                ds.fit_rotations()
                launches += 1
        ds.bond_stress(with_force=False, with_ratio=fetch)
        launches += 1
        return it, launches, worst

    # one step assembles the system, the autotuner picks the inner-solve launch
    # configuration from it, then the warm-up steps run with that choice
    step()
    tuning = ds.autotune(precision)
    for _ in range(args.warmup):
        step()

    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    total_ms, total_it, total_launch, worst = 0.0, 0, 0, 0.0
    for k in range(args.steps):
        with torch.cuda.stream(ext):
            flush.fill_(k & 0xFF)  # L2 flush between timed steps
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        it, launches, w = step()
        e1.record(ext)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        total_it += it
        total_launch += launches
        worst = max(worst, w)
    torch.cuda.synchronize()
    clk = clocks.stop()
    if dist:
        dist.barrier()

    # aggregate: max device time over ranks, summed work
    dof_iters = float(free_dof) * total_it
    job_ms, job_dof_iters, job_solves = combine_ranks(total_ms, dof_iters, float(passes * args.steps),
                                                      dist, "cuda")
    value = job_dof_iters / (job_ms / 1000.0)

    # kernel roofline, CUDA events on the scene stream (cold: L2 flushed before the launch)
    cold = ds.kernel_times(precision, reps=20, flush_ptr=flush.data_ptr(), flush_bytes=flush.numel())
    warm = ds.kernel_times(precision, reps=20)
    peak, peak_kind = measured_peak()
    prof = profiled_traffic() or {}
    fp64 = precision == N.PRECISION_FP64
    mv_bytes = BYTES_PER_REV["matvec_f64" if fp64 else "matvec_f32"] * active
    up_bytes = BYTES_PER_REV["update_f64" if fp64 else "update_f32"] * active
    streaming = {"matvec_us_cold_l2": cold["matvec_us"], "matvec_us_warm_l2": warm["matvec_us"],
                 "update_us_cold_l2": cold["update_us"], "update_us_warm_l2": warm["update_us"],
                 "matvec_gbs_cold_l2": mv_bytes / (cold["matvec_us"] * 1e-6) / 1e9,
                 "update_gbs_cold_l2": up_bytes / (cold["update_us"] * 1e-6) / 1e9}
    if not args.no_large_matvec:
        streaming["large_lattice"] = large_matvec(ctx, flush, peak)
    batched = None
    if not args.no_batched_ratio:
        # a smaller batch of the batched workload, so its ratio to the plain FP64
        # single-scene form is in the default line
        from vxsim import batched as B
        small = B.batched_scenes(args.batched_ratio_scenes, seed=2024 + rank)
        batched = batched_vs_fp64(ctx, local, small, 3, 2, args.tolerance, args.max_iterations)
        batched["workload"] = (f"batched {len(small)} box-union scenes (edge log-uniform 8-48), one pass each, "
                               f"3 timed batched solves")
    if cold["persistent_iter_us"] > 0:
        # the whole inner solve is one persistent launch: algorithmic bytes of a
        # streamed iteration (matvec + update + direction) per iteration time
        it_bytes = (BYTES_PER_REV["matvec_f32"] + BYTES_PER_REV["update_f32"] + BYTES_PER_REV["direction_f32"]) * active
        achieved = it_bytes / (cold["persistent_iter_us"] * 1e-6) / 1e9
        kernel = persistent_kernel_name(cold["persistent_form"], tuning)
        bytes_per_launch = it_bytes * cold["persistent_iterations"]
        launch_us = cold["persistent_iter_us"] * cold["persistent_iterations"]
        traffic = prof.get("persistent_dram_bytes_per_rev_iteration")
        traffic = traffic * scene.n * cold["persistent_iterations"] if traffic else None
        note = ("matrix, z and p stay in shared memory and the vectors in L2 for the whole inner solve, "
                "so HBM traffic per iteration is far below the streamed algorithmic bytes")
    else:
        achieved = streaming["matvec_gbs_cold_l2"]
        kernel = "k_matvec<double>" if fp64 else "k_matvec<float>"
        bytes_per_launch = mv_bytes
        launch_us = cold["matvec_us"]
        # the capture nearest in size: whether the inputs fit L2 changes the bytes per REV
        caps = prof.get("matvec_f32_dram_bytes_per_rev") or []
        near = min(caps, key=lambda c: abs(math.log(c["revs"] / max(scene.n, 1))), default=None)
        traffic = near["bytes_per_rev"] * scene.n if near else None
        note = "streaming matvec launched alone after an L2 flush"
        if fp64:
            traffic = None  # the profiled captures are of the FP32 matvec

    # the step's first pass against the plain FP64 form solved to 1e-12 on the same
    # system (that form matches the C oracle to 1e-10 on the 10^3 wood cube)
    ds.restore_state()
    x0_dev = ds.positions().copy()
    ds.fit_rotations()
    ds.corotational_pass(h, args.tolerance, args.max_iterations, precision=precision,
                         inner_tolerance=args.inner_tolerance)
    dx_mixed = ds.positions() - x0_dev
    ds.restore_state()
    ds.fit_rotations()
    ref = ds.corotational_pass(h, 1e-12, 200000, precision=N.PRECISION_FP64)
    dx_fp64 = ds.positions() - x0_dev
    error_vs_fp64 = {"value": float(np.linalg.norm(dx_mixed - dx_fp64) / max(np.linalg.norm(dx_fp64), 1e-300)),
                     "reference": "displacement of the first pass in the plain FP64 form solved to 1e-12",
                     "reference_true_residual": ref["true_residual"], "reference_iterations": ref["iterations"]}

    # end to end through the C ABI with host buffers (pinned staging inside the library)
    e2e = None
    if not args.no_e2e:
        # the step's inputs and outputs in page-locked host memory, as an engine
        # keeps its staging buffers; the library copies them by DMA
        torch_types = {np.float64: torch.float64, np.float32: torch.float32, np.uint8: torch.uint8}

        def pinned(a, dtype):
            t = torch.empty(np.asarray(a).size, dtype=torch_types[dtype], pin_memory=True)
            view = t.numpy()
            view[:] = np.asarray(a, dtype).reshape(-1)
            return t, view

        keep = [pinned(scene.position, np.float64), pinned(scene.rotation, np.float64), pinned(pred, np.float64),
                pinned(scene.target_mask, np.uint8), pinned(scene.target, np.float64),
                pinned(scene.loads, np.float64), pinned(np.zeros(3 * scene.n), np.float64),
                pinned(np.zeros(3 * scene.n), np.float32)]
        x0, q0, pred_h, mask_h, target_h, loads_h, x_out, ratio_out = [v for _, v in keep]
        e2e_ms, e2e_it = 0.0, 0
        h2d = scene.n * (24 * 4 + 32 + 1)
        d2h = scene.n * (24 + 12)
        for k in range(max(1, min(args.steps, 3))):
            with torch.cuda.stream(ext):
                flush.fill_(k & 0xFF)
            e0 = torch.cuda.Event(enable_timing=True)
            e1 = torch.cuda.Event(enable_timing=True)
            e0.record(ext)
            ds.set_positions(x0)
            ds.set_rotations(q0)
            ds.set_predicted(pred_h)
            ds.set_targets(mask_h, target_h)
            ds.set_loads(loads_h)
            ds.fit_rotations()
            it = 0
            for p in range(passes):
                st = ds.corotational_pass(h, args.tolerance, args.max_iterations, precision=precision,
                                      inner_tolerance=args.inner_tolerance)
                it += st["iterations"]
                if p + 1 < passes:
                    ds.fit_rotations()
            out = ds.bond_stress(with_force=False, ratio_out=ratio_out)
            xs = ds.positions(out=x_out)
            e1.record(ext)
            e1.synchronize()
            e2e_ms += e0.elapsed_time(e1)
            e2e_it += it
            assert np.all(np.isfinite(xs)) and out["ratio"].shape == (3, scene.n)
        e2e_value = float(free_dof) * e2e_it / (e2e_ms / 1000.0) * world
        e2e = {"value": e2e_value, "unit": "DOF-iter/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
               "ms_per_step": e2e_ms / max(1, min(args.steps, 3))}

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        threads = os.cpu_count() or 1
        rows, dof, it, dt, samples = cpu_reference_rate(scene, h, pred, args.cpu_iterations, threads,
                                                         args.cpu_seconds)
        cpu = {"value": dof * it / dt, "unit": "DOF-iter/s", "cores": threads, "kind": "port",
               "omp_num_threads": threads, "host_cpus": os.cpu_count(),
               "sample": f"{samples} samples of {args.cpu_iterations} iterations ({it} in {dt:.1f} s) of the "
                         f"reference's CPU block-Jacobi PCG loop (f32 restatement, OpenMP, {threads} threads) "
                         f"on pass 0 of this workload, {rows['n']} active REVs"}
        if not args.no_oracle_error:
            # checker: the same first pass solved by the C oracle in FP64
            dx_o, it_o, res_o, t_o = oracle_first_pass(scene, h, pred, 1e-12)
            error_vs_fp64["oracle"] = {
                "value": float(np.linalg.norm(dx_mixed - dx_o) / max(np.linalg.norm(dx_o), 1e-300)),
                "gpu_fp64_vs_oracle": float(np.linalg.norm(dx_fp64 - dx_o) / max(np.linalg.norm(dx_o), 1e-300)),
                "reference": "displacement of the first pass solved by the C oracle (FP64 block-Jacobi PCG) "
                             "to a relative residual of 1e-12",
                "oracle_iterations": it_o, "oracle_residual": res_o, "oracle_seconds": round(t_o, 1)}

    if rank == 0:
        line = {
            "metric": "PCG DOF-iters/s (plain FP64 PCG)" if fp64 else METRIC, "value": value,
            "unit": "DOF-iter/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": job_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if fp64 else "f32+f64", "data": "synthetic",
            "config": workload_config(args, scene, world),
            "solves_per_s": job_solves / (job_ms / 1000.0),
            "iterations_per_solve": total_it / (passes * args.steps),
            "worst_true_residual": worst,
            "error_vs_fp64": error_vs_fp64,
            "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": achieved / peak, "traffic": traffic, "kernel": kernel,
                         "bytes_per_launch": bytes_per_launch, "launch_us": launch_us,
                         "peak_source": f"{peak_kind} hbm_gbs", "note": note},
            "streaming_kernels": streaming,
            "batched": batched,
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": total_launch,
            "tuning": {"choice": N.tune_label(tuning["kernel"], tuning["blocks_per_sm"]),
                       "us_per_iteration": tuning["us_per_iteration"],
                       "candidates_us": {N.tune_label(k, b): round(us, 2) for k, b, us in tuning["candidates"]}},
            "clocks": clk,
        }
        print(json.dumps(line), flush=True)
    ds.close()
    ctx.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return 0


def batched_vs_fp64(ctx, local, scenes, steps, warmup, tolerance, max_iterations, fp64_sample=None,
                    kernel=None):
    """The batched form (every scene resident in one pool, one corotational pass
    each, FP32 inner PCG in FP64 refinement) timed over `steps` batched solves
    with CUDA events on the pool's stream and an L2 flush before each, against
    the same scenes solved one at a time in the plain FP64 single-scene form
    (each scene warmed once, then timed once)."""
    import torch
    from vxsim import batched as B
    from vxsim import native as N
    bs = B.BatchedSolve(ctx, scenes, tolerance=tolerance, max_iterations=max_iterations,
                        kernel=N.KERNEL_AUTO if kernel is None else kernel)
    ext = torch.cuda.ExternalStream(bs.stream_ptr, device=torch.device("cuda", local))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")
    for _ in range(warmup):
        bs.solve()
    torch.cuda.synchronize()
    total_ms, dof_iters, worst, launches = 0.0, 0.0, 0.0, 0
    for k in range(steps):
        with torch.cuda.stream(ext):
            flush.fill_(k & 0xFF)
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        status, stats = bs.solve()
        e1.record(ext)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        assert status == N.VX_OK, status
        for st in stats:
            dof_iters += 3.0 * st["active"] * st["iterations"]
            worst = max(worst, st["true_residual"])
        launches += 1 + max(st["kernel_launches"] for st in stats)
    bs.close()
    sample = scenes if fp64_sample is None else scenes[:fp64_sample]
    ss = B.SingleSceneSolves(ctx, sample, tolerance=tolerance, max_iterations=max_iterations)
    for k in range(len(sample)):  # warm every scene: its graph capture stays out of the timed solves
        ss.solve(k)
    fp64_ms, fp64_worst = 0.0, 0.0
    for k in range(len(sample)):
        ek = torch.cuda.ExternalStream(ss.devs[k].stream_ptr, device=torch.device("cuda", local))
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(ek)
        st = ss.solve(k)
        e1.record(ek)
        e1.synchronize()
        fp64_ms += e0.elapsed_time(e1)
        fp64_worst = max(fp64_worst, st["true_residual"])
    ss.close()
    solves_per_s = len(scenes) * steps / (total_ms / 1000.0)
    fp64_solves_per_s = len(sample) / (fp64_ms / 1000.0)
    return {"solves_per_s": solves_per_s, "ms_per_step": total_ms / steps,
            "dof_iters_per_s": dof_iters / (total_ms / 1000.0), "worst_true_residual": worst,
            "revs_total": sum(s.n for s in scenes), "scenes": len(scenes), "gpu_launches": launches,
            "fp64_single_scene": {"solves_per_s": fp64_solves_per_s, "scenes_timed": len(sample),
                                  "worst_true_residual": fp64_worst,
                                  "form": "vx_corotational_pass, VX_PRECISION_FP64, one scene at a time"},
            "speedup_vs_fp64_single_scene": solves_per_s / fp64_solves_per_s}


def batched_arm(args):
    """The batched workload (512 box-union scenes, one corotational pass each, FP32 inner PCG in FP64
    refinement to 1e-8, solved together in one pool) against the same scenes solved one at a time in the
    plain FP64 single-scene form. Prints one JSON line; value = batched solves/s."""
    import torch
    from vxsim import batched as B
    from vxsim import native as N
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    scenes = B.batched_scenes(args.scenes, seed=2024 + rank)
    ctx = N.Context(local)
    clocks = ClockSampler(local)
    clocks.start()
    kernel = {"auto": N.KERNEL_AUTO, "persistent": N.KERNEL_PERSISTENT,
              "streaming": N.KERNEL_STREAMING}[args.pool_kernel]
    out = batched_vs_fp64(ctx, local, scenes, args.steps, args.warmup, args.tolerance, args.max_iterations,
                          args.fp64_sample, kernel)
    clk = clocks.stop()
    if rank == 0:
        print(json.dumps({
            "metric": "batched solves/s (one corotational pass per scene, FP32 inner PCG in FP64 refinement "
                      "to 1e-8)",
            "value": out["solves_per_s"] * world, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": out["ms_per_step"], "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64", "data": "synthetic",
            "config": {"workload": f"batched {len(scenes)} box-union scenes, edge log-uniform 8-48",
                       "scenes": len(scenes), "revs_total": out["revs_total"], "tolerance": args.tolerance,
                       "inner_solve": args.pool_kernel,
                       "l2": "256 MiB buffer written between timed steps", "parallelism": f"replicas{world}"},
            "dof_iters_per_s": out["dof_iters_per_s"],
            "worst_true_residual": out["worst_true_residual"],
            "fp64_single_scene": out["fp64_single_scene"],
            "speedup_vs_fp64_single_scene": out["speedup_vs_fp64_single_scene"],
            "gpu_launches": out["gpu_launches"], "clocks": clk,
        }), flush=True)
    ctx.close()
    return 0


def served_arm(args):
    """The served workload through vx_server: Poisson arrivals of scene-step requests, continuous
    batching, admission by an 80% HBM pool. Prints one JSON line; value = solves/s over the run."""
    from vxsim import native as N
    from vxsim import served as V
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    ctx = N.Context(local)
    clocks = ClockSampler(local)
    clocks.start()
    out = V.run_served(ctx, rate=args.rate, duration=args.window, steps=args.request_steps, max_slots=args.slots,
                       lanes=args.lanes,
                       drain=args.drain, tolerance=args.tolerance, seed=77 + rank)
    clk = clocks.stop()
    st = out["stats"]
    # the single-scene forms on the requests' own steps: each template stepped
    # alone, weighted by how often the request stream picked it
    fp64 = None
    if not args.no_fp64_compare:
        import numpy as np
        picks = np.bincount(out["template_picks"], minlength=len(out["template_scenes"]))
        served_rate = st["solves"] / out["wall_s"]
        fp64 = {}
        for name, prec in (("fp64", N.PRECISION_FP64), ("mixed", N.PRECISION_MIXED)):
            rows = V.single_scene_step_rate(ctx, out["template_scenes"], prec, steps=4, tolerance=args.tolerance)
            per_solve = float(np.dot(picks, [r["seconds"] / max(r["solves"], 1) for r in rows]) / max(picks.sum(), 1))
            fp64[name] = {"solves_per_s": 1.0 / per_solve,
                          "worst_residual": max(r["worst_residual"] for r in rows),
                          "per_template_ms_per_solve": [round(1000 * r["seconds"] / max(r["solves"], 1), 2)
                                                        for r in rows]}
        fp64["form"] = ("each template scene alone (vx_scene_step), its first 4 request steps (blade, contact, "
                        "fracture), solves weighted by the request mix")
        fp64["speedup_served_vs_fp64"] = served_rate / fp64["fp64"]["solves_per_s"]
    if rank == 0:
        print(json.dumps({
            "metric": "served solves/s (Poisson scene-step requests, continuous batching, FP32 inner PCG in FP64 "
                      "refinement to 1e-8)",
            "value": st["solves"] / out["wall_s"] * world, "unit": "solves/s", "n_gpus": world,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32+f64",
            "data": "synthetic",
            "config": {"workload": "served: wood blocks cut by a driven iron blade through contact and fracture",
                       "arrival_rate_per_s": out["arrival_rate"], "arrival_window_s": out["arrival_window_s"],
                       "steps_per_request": out["steps_per_request"], "max_slots": args.slots,
                       "dof_range": out["dof_range"], "hbm_budget": 0.8, "blade": out["blade"],
                       "lanes": out["lanes"],
                       "parallelism": f"replicas{world}"},
            "p50_step_ms": st["p50_step_ms"], "p99_step_ms": st["p99_step_ms"], "max_step_ms": st["max_step_ms"],
            "request_latency_s": out["request_latency_s"], "fp64_single_scene": fp64,
            "scene_steps_per_s": st["scene_steps"] / out["wall_s"],
            "requests": out["requests"], "completed": out["completed"], "not_converged": out["not_converged"],
            "queued_at_end": st["queued"], "resident_at_end": st["resident"], "rounds": st["rounds"],
            "busy_fraction": st["busy_s"] / max(out["wall_s"], 1e-9), "mean_queued_s": out["mean_queued_s"],
            "worst_residual_completed": out["worst_residual"], "worst_residual_all_steps": st["worst_residual"],
            "not_converged_scene_steps": st["not_converged"], "wall_s": out["wall_s"],
            "pool_revs": st["pool_revs"], "pool_gb": st["pool_bytes"] / 1e9, "clocks": clk,
        }), flush=True)
    ctx.close()
    return 0


def contact_arm(args):
    """Contact projection (collision::project) on the device: a 64^3 iron block
    (262,144 REVs) standing on its kinematic bottom layer, which is not bonded
    to it, after the prediction of one 0.25 ms substep under gravity (the block
    has moved g h^2 into the layer). One step = one vx_contact_project call:
    the broadphase over every REV's swept box, the intact-lattice filter and the
    ordered projection sweeps. Value = candidate pairs per second."""
    import torch
    from vxsim import materials as M
    from vxsim import native as N
    from vxsim import scenes as S

    local = int(os.environ.get("LOCAL_RANK", "0"))
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    torch.cuda.set_device(local)
    edge = args.edge or 64
    cells = S.grid_cells(edge, edge, edge)
    scene = S.from_cells(cells, M.component_id("iron"), M.table(), kinematic=(cells[:, 2] == 0))
    h = 1e-3 / 4
    g = 9.81
    prev = scene.position.copy()
    pos = prev.copy()
    pos[cells[:, 2] > 0, 2] -= g * h * h
    ctx = N.Context(local)
    ds = N.DeviceScene(ctx, scene)
    ext = torch.cuda.ExternalStream(ds.stream_ptr, device=torch.device("cuda", local))
    flush = torch.empty(256 << 20, dtype=torch.uint8, device=f"cuda:{local}")

    def reset():
        ds.write_field(N.FIELD_POSITION, pos)
        ds.write_field(N.FIELD_PREVIOUS, prev)

    for _ in range(args.warmup):
        reset()
        st = ds.contact_project()
    torch.cuda.synchronize()
    clocks = ClockSampler(local)
    clocks.start()
    total_ms, launches, stats = 0.0, 0, None
    for k in range(args.steps):
        reset()
        with torch.cuda.stream(ext):
            flush.fill_(k & 0xFF)
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        stats = ds.contact_project()
        e1.record(ext)
        e1.synchronize()
        total_ms += e0.elapsed_time(e1)
        launches += stats["launches"]
    clk = clocks.stop()
    ms = total_ms / args.steps
    # end to end: host positions and previous positions in (page-locked), the
    # projection, contacts and positions out
    def pinned(a):
        t = torch.empty(a.size, dtype=torch.float64, pin_memory=True)
        v = t.numpy()
        v[:] = a.reshape(-1)
        return t, v

    keep = [pinned(pos), pinned(prev), pinned(np.zeros(pos.size))]
    pos_h, prev_h, out_h = (v for _, v in keep)
    e2e_ms = 0.0
    reps = max(1, min(args.steps, 3))
    for k in range(reps):
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(ext)
        ds.set_positions(pos_h)
        ds.set_previous(prev_h)
        ds.contact_project()
        c = ds.contacts()
        x = ds.positions(out=out_h)
        e1.record(ext)
        e1.synchronize()
        e2e_ms += e0.elapsed_time(e1)
    e2e_ms /= reps
    cpu = None
    if rank == 0 and not args.no_cpu_baseline:
        import pyoracle as O
        t0 = time.perf_counter()
        _, _, oc, ost = O.contact_project(pos, prev, scene.position, scene.kinematic, scene.mass.astype(np.float64),
                                          scene.neighbor)
        dt = time.perf_counter() - t0
        assert ost["pairs"] == stats["pairs"] and len(oc) == stats["contacts"]
        cpu = {"value": ost["candidates"] / dt, "unit": "candidate pairs/s", "cores": 1, "kind": "port",
               "sample": "one collision::project call of this workload in the C restatement (FP64, serial as "
                         f"the reference's project), {dt:.2f} s"}
    if rank == 0:
        print(json.dumps({
            "metric": "contact projection candidate pairs/s (collision::project: broadphase, intact-lattice "
                      "filter, ordered sweeps)",
            "value": stats["candidates"] / (ms / 1000.0) * world, "unit": "candidate pairs/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"contact: iron block {edge}^3 on its kinematic layer after one substep",
                       "revs": scene.n, "candidates": stats["candidates"], "pairs": stats["pairs"],
                       "stored_pairs": stats["stored"], "contacts": stats["contacts"], "sweeps": stats["sweeps"],
                       "live_max": stats["live_max"],
                       "l2": "256 MiB buffer written between timed steps", "parallelism": f"replicas{world}"},
            "e2e": {"value": stats["candidates"] / (e2e_ms / 1000.0) * world, "unit": "candidate pairs/s",
                    "h2d_bytes_per_step": 2 * 24 * scene.n, "d2h_bytes_per_step": 24 * scene.n + 13 * len(c),
                    "ms_per_step": e2e_ms},
            "cpu_baseline": cpu, "gpu_launches": launches, "clocks": clk,
        }), flush=True)
    ds.close()
    ctx.close()
    return 0


def main():
    args = parse()
    if args.impl == "reference":
        return reference_arm(args)
    if args.workload == "batched":
        return batched_arm(args)
    if args.workload == "served":
        return served_arm(args)
    if args.workload == "contact":
        return contact_arm(args)
    return our_arm(args)


if __name__ == "__main__":
    sys.exit(main())

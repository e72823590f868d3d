#!/usr/bin/env python
"""Throughput of the plain 3D FDTD loop on B200: Gcell-updates/s and the HBM roofline fraction.

Workload (lightsmith's plain-FDTD throughput case): a 640^3 FP32 grid, 16-cell CPML on every face,
i.i.d. permittivity uniform in [1, 12.25] drawn from a seed, a Gaussian point-current pulse at the centre,
a 16-frequency running DFT on the centre z plane. One bench step is one chunk: dft_stride FDTD time steps
plus one DFT sample (lightsmith's unit of work, ``Engine.chunk``), replayed as a CUDA graph.

    python bench.py [--gpus N --steps K --warmup W] [--impl b200|reference] [--n 640]

``--impl reference`` times lightsmith's own CPU FDTD (its ``Engine`` from the reference install in
``baseline/_ref``, float64 as lightsmith runs on CPUs, through PyTorch on all host threads, with its NumPy path
beside it) on a 128^3 sample of the same workload. Under torchrun each rank runs an
independent replica (the plain solver does not shard) and rank 0 prints one JSON line.
"""

from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, HERE)

METRIC = "FDTD Gcell-updates/s"
UNIT = "Gcell-updates/s"
CPU_SAMPLE_N = 128
# algorithmic bytes of one FP32 cell update with isotropic eps: E and H read once and written once (6 + 6
# values) and one coefficient read; each CPML (cell, axis) pair adds 4 psi values read and written
BYTES_PER_CELL = (12 + 1) * 4
BYTES_PER_CPML_PAIR = 4 * 2 * 4


def _args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--n", type=int, default=640)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--variant", type=int, default=-1,
                    help="0 in-place (vector) kernels, 1 fused pass; -1: pick the faster on this GPU (tuner)")
    ap.add_argument("--tile-y", type=int, default=8, help="fused pass: tile rows along y")
    ap.add_argument("--planes", type=int, default=0, help="fused pass: x planes per CTA (0: chosen per grid)")
    ap.add_argument("--stages", type=int, default=4, help="fused pass: x planes in the copy ring")
    ap.add_argument("--workload", default="throughput", choices=["throughput", "sweep", "adjoint", "clusters",
                                                                 "sphere", "setup"],
                    help="sweep: the batched oblique-incidence sweep (96 Bloch-periodic runs) against the same "
                         "runs one after another; adjoint: the slab device's gradient against its forward run; "
                         "clusters: forward + gradient over dispersive sphere clusters, with FP64 errors; sphere: "
                         "the whole 129^3 dispersive-sphere solve from lightsmith's own plan, with its cross "
                         "sections against lightsmith's FP64 CPU solve; setup: that sphere's meshing by lightsmith "
                         "on the host and on the GPU")
    ap.add_argument("--runs", type=int, default=96, help="sweep: number of runs")
    ap.add_argument("--sweep-steps", type=int, default=3000, help="sweep: FDTD steps per run")
    ap.add_argument("--instances", type=int, default=24, help="clusters: number of instances")
    ap.add_argument("--cluster-steps", type=int, default=2000, help="clusters: FDTD steps per instance")
    ap.add_argument("--no-forms", action="store_true",
                    help="the default line without its records of the other forms (sphere solve, batched sweep, "
                         "adjoint, clusters)")
    ap.add_argument("--form-instances", type=int, default=4, help="cluster instances in the default line's record")
    return ap.parse_args()


def _peak():
    try:
        with open(os.path.join(HERE, "MEASURED_PEAKS.json")) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return 6650.0, "fallback"


def _ncu_traffic(kernel: str, grid, shape_tuple):
    """DRAM bytes (read + write) of one step of ``kernel`` on ``grid`` in kernel variant ``shape_tuple[0]``
    (the launches of one step summed: the lean pass split by class of CTA box, which tile rows 8 and a ring of
    4 select, takes five), as one ncu capture of the same kernel on the same grid recorded them
    (``profiles/ncu_traffic.json``, each record with the command that made it): (bytes, source) or
    (None, None) without a matching record."""
    split = int(shape_tuple[0]) == 4 and int(shape_tuple[1]) == 8 and int(shape_tuple[3]) == 4
    try:
        with open(os.path.join(HERE, "profiles", "ncu_traffic.json")) as f:
            records = json.load(f)
    except (OSError, ValueError):
        return None, None
    for r in records:  # the same kernel, grid and kernel variant (planes per CTA change the halo re-reads only)
        if (r.get("kernel") == kernel and list(r.get("grid", [])) == list(grid) and
                int(r.get("variant", -1)) == int(shape_tuple[0]) and bool(r.get("split", False)) == split):
            return float(r["dram_bytes_read"]) + float(r["dram_bytes_write"]), \
                f"ncu capture of one step of the same kernel and grid: {r['command']}"
    return None, None


class Clocks:
    """nvidia-smi samples (every 200 ms) of one GPU while the timed region runs."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
    NAMES = ("hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap")

    def __init__(self, gpu_id):
        self.proc = None
        cmd = ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits", "-lms", "200"]
        if gpu_id:
            cmd += ["-i", gpu_id]
        try:
            self.proc = subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except OSError:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
            out, _ = self.proc.communicate()
        sm, mx, reasons = [], [], set()
        for line in out.strip().splitlines():
            parts = [p.strip() for p in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                mx.append(float(parts[2]))
            except ValueError:
                continue
            for name, flag in zip(self.NAMES, parts[5:9]):
                if flag.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": statistics.median(sm), "sm_max_mhz": max(mx), "reasons": sorted(reasons),
                "samples": len(sm)}


def _gpu_uuid(torch, dev):
    try:
        u = str(torch.cuda.get_device_properties(dev).uuid)
        return u if u.startswith("GPU-") else "GPU-" + u
    except Exception:  # noqa: BLE001 (older torch)
        return None


def cpu_sample(n: int, chunks: int, warmup: int, threads: int):
    """The oracle port (float64, as lightsmith runs on CPUs) on an n^3 sample of the workload, used only where
    lightsmith itself is not installed: (Gcell-updates/s, seconds, stride)."""
    from lightsmith_b200.workloads import throughput_plan
    from oracle.engine import OracleEngine

    plan = throughput_plan(n, max_steps=400 * (chunks + warmup + 2), single=False, seed=1)
    eng = OracleEngine(plan, threads=threads)
    for _ in range(warmup):
        eng.chunk()
    t0 = time.perf_counter()
    for _ in range(chunks):
        eng.chunk()
    dt = time.perf_counter() - t0
    eng.close()
    cells = n ** 3
    return cells * plan["stride"] * chunks / dt / 1e9, dt, plan["stride"]


REF_INSTALL = os.path.join(HERE, "baseline", "_ref")


def _lightsmith_available() -> bool:
    """lightsmith itself (the reference install, ``baseline/install_ref.py``) on sys.path."""
    if not os.path.isdir(os.path.join(REF_INSTALL, "lightsmith")):
        return False
    if REF_INSTALL not in sys.path:
        sys.path.insert(0, REF_INSTALL)
    try:
        import lightsmith  # noqa: F401
    except Exception:  # noqa: BLE001 (a broken install counts as none)
        return False
    return True


def reference_sample(n: int, chunks: int, warmup: int, threads: int, device: str = "torch-cpu"):
    """lightsmith's own FDTD engine (``backends/_fdtd/engine.py:Engine``, with its ``PointDipole``,
    ``DFTMonitor`` and ``PMLSpec``) on an n^3 sample of the throughput workload, float64 as lightsmith runs on
    CPUs, on ``device`` ("torch-cpu": PyTorch on ``threads`` host threads; "cpu": NumPy, whose ufuncs use one
    core): (Gcell-updates/s, seconds, stride)."""
    from lightsmith.backends._fdtd.emission import PointDipole
    from lightsmith.backends._fdtd.engine import DFTMonitor, Engine, PMLSpec
    from lightsmith.device import resolve_device

    from lightsmith_b200.workloads import plane_monitor, throughput_band

    if device == "torch-cpu":
        import torch

        torch.set_num_threads(threads)
    shape = (n, n, n)
    dx = 20.0
    dt, om, omega_c, omega_half, stride = throughput_band(dx)
    inv = 1.0 / np.random.default_rng(1).uniform(1.0, 12.25, size=shape)
    inv3 = np.ascontiguousarray(np.broadcast_to(inv, (3,) + shape))
    steps = stride * (chunks + warmup + 2)
    dip = PointDipole(shape=shape, origin=np.zeros(3), dx=dx, dt=dt, pos=(np.asarray(shape) // 2) * dx + 0.37 * dx,
                      pdir=(0.0, 0.0, 1.0), inv_eps=inv3, omega_c=omega_c, omega_half=omega_half, max_steps=steps)
    m = plane_monitor(shape, n // 2, om, energy=1)
    mon = DFTMonitor(m.omega, m.e_idx, m.h_idx1, m.h_idx2, energy=1)
    pml = PMLSpec(cells=((16, 16),) * 3, alpha_max=0.05 * 2 * np.pi / 2000.0, eps_ref=1.0)
    eng = Engine(resolve_device(device), shape=shape, dx=dx, dt=dt, single=False, inv_eps=inv3, groups=[], pml=pml,
                 sources=[dip], monitors=[mon], dft_stride=stride)
    for _ in range(warmup):
        eng.chunk()
    t0 = time.perf_counter()
    for _ in range(chunks):
        eng.chunk()
    secs = time.perf_counter() - t0
    return n ** 3 * stride * chunks / secs / 1e9, secs, stride


def cpu_baseline_record(n: int, chunks: int, warmup: int, threads: int, numpy_chunks: int = 1) -> dict:
    """The CPU baseline: lightsmith's own engine on torch-cpu (all threads) with its NumPy path beside it; the
    oracle port where lightsmith is not installed."""
    if _lightsmith_available():
        v, secs, st = reference_sample(n, chunks, warmup, threads, "torch-cpu")
        rec = {"value": v, "unit": UNIT, "cores": threads, "kind": "reference",
               "sample": f"{n}^3 grid of the same workload (CPML 16, random eps, centre dipole, 16-frequency DFT "
                         f"plane), {chunks} chunks of {st} steps after {warmup}, lightsmith 0.3.0's own Engine on "
                         f"device 'torch-cpu', float64, {threads} threads ({secs:.1f} s)", "seconds": secs}
        if numpy_chunks:
            vn, sn, _ = reference_sample(n, numpy_chunks, 0, threads, "cpu")
            rec["numpy_fp64"] = {"value": vn, "unit": UNIT, "cores": 1,
                                 "sample": f"the same engine on device 'cpu' (NumPy float64; its ufuncs run on one "
                                           f"core of {threads}), {numpy_chunks} chunk(s) ({sn:.1f} s)"}
        return rec
    v, secs, st = cpu_sample(n, chunks, warmup, threads)
    return {"value": v, "unit": UNIT, "cores": threads, "kind": "port",
            "sample": f"{n}^3 grid of the same workload, {chunks} chunks of {st} steps after {warmup}, NumPy "
                      f"float64 oracle port on {threads} threads ({secs:.1f} s; lightsmith itself not installed)",
            "seconds": secs}


def _threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def run_reference(args):
    """lightsmith's own CPU FDTD on the host cores: each bench step is one chunk (stride steps + one DFT sample)
    of a 128^3 sample of the throughput workload, on lightsmith's engine through PyTorch on all host threads
    (float64, as lightsmith runs on CPUs); the oracle port stands in only where lightsmith is not installed."""
    if int(os.environ.get("RANK", "0")) != 0:
        return
    threads = _threads()
    rec = cpu_baseline_record(CPU_SAMPLE_N, args.steps, args.warmup, threads, numpy_chunks=1)
    value = rec["value"]
    secs = rec["seconds"]
    out = {"metric": METRIC, "value": value, "unit": UNIT, "impl": "reference", "n_gpus": args.gpus,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * secs / max(args.steps, 1),
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
           "config": {"workload": f"plain FDTD throughput, {CPU_SAMPLE_N}^3 CPU sample of the 640^3 case (CPML 16, "
                                  "i.i.d. eps in [1, 12.25], centre dipole pulse, 16-frequency DFT on one plane)",
                      "grid": [CPU_SAMPLE_N] * 3, "dx_nm": 20.0},
           "cpu_baseline": rec,
           "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(out), flush=True)


def run_b200(args):
    import numpy as np
    import torch

    from lightsmith_b200.engine import Engine
    from lightsmith_b200.workloads import cells_in_cpml, throughput_band, throughput_plan

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300), device_id=dev)

    n = args.n
    shape = (n, n, n)
    K, W = args.steps, args.warmup
    R = max(1, min(K, 6))  # chunks of the kernel-timing pass
    _, _, _, _, stride = throughput_band()
    from lightsmith_b200.tune import CANDIDATES

    total_chunks = W + 2 * K + R + 2 + 3 * len(CANDIDATES) + 2  # the tuner's eager chunks (3 per candidate) too
    gen = torch.Generator(device=dev)
    gen.manual_seed(1234)
    inv = 1.0 / (torch.rand(shape, generator=gen, device=dev, dtype=torch.float32) * 11.25 + 1.0)
    plan = throughput_plan(n, inv_eps=inv, max_steps=stride * total_chunks + 8, single=True)
    eng = Engine.from_plan(plan, device=dev)
    if args.variant < 0:
        from lightsmith_b200.tune import tune_engine

        tuned, _ = tune_engine(eng)
        variant = tuned[0]
    else:
        tuned = (args.variant, args.tile_y, args.planes, args.stages)
        variant = args.variant
        eng.set_tuning(*tuned)
    inv_host = torch.empty(shape, dtype=torch.float32, pin_memory=True)
    inv_host.copy_(inv)
    del inv, plan["inv_eps"]
    torch.cuda.empty_cache()
    cells = n ** 3

    eng.chunk(W, use_graph=True)
    torch.cuda.synchronize(dev)
    if dist:
        dist.barrier()
    clocks = Clocks(_gpu_uuid(torch, dev)) if rank == 0 else None
    time.sleep(0.3 if clocks else 0.0)
    start, end = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    start.record(eng.stream)
    eng.chunk(K, use_graph=True)
    end.record(eng.stream)
    torch.cuda.synchronize(dev)
    ms = start.elapsed_time(end)
    if dist:
        dist.barrier()
    clk = clocks.stop() if clocks else None
    t = torch.tensor([ms], device=dev, dtype=torch.float64)
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * cells * stride * K / (ms_max / 1e3) / 1e9

    # the bulk Yee kernels alone: CUDA events around each launch on the engine's stream
    bulk_ms, bulk_launches = eng.chunk_timed(R)
    steps_timed = R * stride
    step_ms = bulk_ms / steps_timed
    alg_bytes = cells * BYTES_PER_CELL + cells_in_cpml(eng.plan) * BYTES_PER_CPML_PAIR
    achieved = alg_bytes / (step_ms / 1e3) / 1e9
    peak, peak_kind = _peak()
    traffic, traffic_source = _ncu_traffic("k_fused_pml", shape, tuned)

    # end to end through the C ABI with host buffers: permittivity from pinned host memory, K chunks, the DFT
    # accumulators and the energy back to pinned host memory
    acc = [m["acc_e"] for m in eng.monitors] + [m["acc_h"] for m in eng.monitors if m["acc_h"] is not None]
    acc_host = [torch.empty(a.shape, dtype=a.dtype, pin_memory=True) for a in acc]
    energy_host = torch.empty(2, dtype=torch.float64, pin_memory=True)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    with torch.cuda.stream(eng.stream):
        e0.record(eng.stream)
        eng.load_inv_eps(inv_host)
        eng.chunk(K, use_graph=True)
        for h, d in zip(acc_host, acc):
            h.copy_(d, non_blocking=True)
        energy_host.copy_(eng.energy, non_blocking=True)
        e1.record(eng.stream)
    e1.synchronize()
    e2e_ms = e0.elapsed_time(e1)
    te = torch.tensor([e2e_ms], device=dev, dtype=torch.float64)
    if dist:
        dist.all_reduce(te, op=dist.ReduceOp.MAX)
    e2e_value = world * cells * stride * K / (float(te.item()) / 1e3) / 1e9
    h2d = inv_host.numel() * 4
    d2h = sum(a.numel() * a.element_size() for a in acc) + 16
    finite = bool(np.isfinite(energy_host.numpy()).all())
    launches = eng.launches_per_chunk() * K
    eng_fused = eng.fused
    eng_tma = eng.uses_tma

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu = cpu_baseline_record(CPU_SAMPLE_N, 4, 1, _threads(), numpy_chunks=1)
    eng.close()
    del eng
    torch.cuda.empty_cache()
    other = forms(args) if (rank == 0 and world == 1 and not args.no_forms) else None
    if rank == 0:
        out = {"metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": K, "warmup": W,
               "ms_per_step": ms_max / K, "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
               "dtype": "f32", "data": "synthetic",
               "config": {"workload": f"plain FDTD throughput: {n}^3 FP32 grid, 16-cell CPML on all faces, i.i.d. "
                                      "eps in [1, 12.25], centre dipole pulse, 16-frequency DFT on one plane",
                          "grid": list(shape), "cpml_cells": 16, "dft_freqs": 16, "dft_stride": stride,
                          "step": f"one chunk = {stride} FDTD steps + one DFT sample, CUDA graph replay",
                          "l2": "inputs larger than L2 (about 8 GB of state per replica)",
                          "parallelism": f"{world} independent replicas" if world > 1 else "single GPU",
                          "launch_shape": {"variant": tuned[0], "tile_y": tuned[1],
                                           "planes": tuned[2] or "per grid", "ring": tuned[3]},
                          "variant": {0: "in-place H and E kernels", 1: "fused single pass",
                                      2: "in-place four-node H and E kernels",
                                      3: "fused single pass over the interior box + CPML/wall shell kernels",
                                      4: "fused single pass with lean CPML terms"}[variant],
                          "copy_engine": ("TMA" if eng_tma else "cp.async") if variant in (1, 3, 4) else None},
               "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                            "frac": achieved / peak, "peak_source": peak_kind,
                            "traffic": traffic, "traffic_source": traffic_source,
                            "kernel": "bulk Yee update (H and E with their CPML terms), per FDTD step",
                            "alg_bytes_per_step": alg_bytes, "kernel_ms_per_step": step_ms,
                            "bulk_launches_timed": bulk_launches},
               "cpu_baseline": cpu,
               "e2e": {"value": e2e_value, "unit": UNIT, "h2d_bytes_per_step": h2d / K, "d2h_bytes_per_step": d2h / K,
                       "fields_finite": finite},
               "gpu_launches": launches, "clocks": clk}
        if other is not None:
            out["forms"] = other
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


def run_sweep(args):
    """The batched Bloch sweep: ``--runs`` oblique runs of a periodic metasurface cell (10 nm grid, period
    U(300, 600) nm, so 30-60 x 30-60 x 200 cells, complex64 fields), ``--sweep-steps`` steps each. One bench
    step is one launch of the persistent kernel in which every run advances (sweep steps / (W + K)) steps,
    replayed as a CUDA graph; the same runs are then stepped one after another by their own engines (chunks
    replayed as CUDA graphs), and the two sets of DFT accumulators are compared."""
    import numpy as np
    import torch

    from lightsmith_b200.batch import BlochBatch
    from lightsmith_b200.engine import Engine
    from lightsmith_b200.workloads import metasurface_sweep

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    K, W = args.steps, args.warmup
    per_launch = max(1, args.sweep_steps // (K + W))
    plans = metasurface_sweep(args.runs, seed=2024, steps=args.sweep_steps + 8)
    lasts = [(per_launch * (K + W) // p["stride"]) * p["stride"] for p in plans]  # whole chunks per run
    cells = [int(np.prod(p["shape"])) for p in plans]
    cell_steps = sum(c * l for c, l in zip(cells, lasts))
    engines = [Engine.from_plan(p, device=dev) for p in plans]
    batch = BlochBatch(engines, lasts)
    batch.run(per_launch, W, use_graph=True)  # warm-up launches (the runs advance)
    done_warm = [min(W * per_launch, last) for last in lasts]
    clocks = Clocks(_gpu_uuid(torch, dev))
    time.sleep(0.3)
    t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize(dev)
    t0.record(batch.stream)
    batch.run(per_launch, K, use_graph=True)
    t1.record(batch.stream)
    torch.cuda.synchronize(dev)
    ms_batch = t0.elapsed_time(t1)
    clk = clocks.stop()
    timed_cell_steps = sum(c * (last - w) for c, last, w in zip(cells, lasts, done_warm))
    acc_b = [[m["acc_e"].cpu().numpy() for m in e.monitors] for e in engines]
    ctas = batch.ctas
    batch.close()
    for e in engines:
        e.close()
    del engines, batch
    torch.cuda.empty_cache()

    # the same runs one after another, each its own engine and CUDA-graph chunks
    ms_seq, worst = 0.0, 0.0
    for p, last, acc in zip(plans, lasts, acc_b):
        e = Engine.from_plan(p, device=dev)
        e.chunk(1, use_graph=True)  # capture; the run continues from there
        torch.cuda.synchronize(dev)
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record(e.stream)
        e.chunk(last // p["stride"] - 1, use_graph=True)
        b.record(e.stream)
        torch.cuda.synchronize(dev)
        ms_seq += a.elapsed_time(b)
        for k, m in enumerate(e.monitors):
            ref = m["acc_e"].cpu().numpy()
            worst = max(worst, float(np.abs(acc[k] - ref).max() / max(np.abs(ref).max(), 1e-300)))
        e.close()
    seq_cell_steps = sum(c * (last - p["stride"]) for c, last, p in zip(cells, lasts, plans))
    value = timed_cell_steps / (ms_batch / 1e3) / 1e9
    seq_value = seq_cell_steps / (ms_seq / 1e3) / 1e9
    out = {"metric": "FDTD Gcell-updates/s (batched Bloch sweep)", "value": value, "unit": UNIT, "n_gpus": 1,
           "steps": K, "warmup": W, "ms_per_step": ms_batch / K, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "c64", "data": "synthetic",
           "config": {"workload": f"{args.runs} Bloch-periodic oblique runs of a TiO2-pillar metasurface cell on "
                                  "SiO2 (10 nm grid, period U(300, 600) nm, 200 z cells, CPML 12 along z), "
                                  "angles, wavelengths and polarisations drawn from a seed",
                      "step": f"one launch of the persistent kernel: every run advances {per_launch} steps",
                      "steps_per_run": lasts[0] if len(set(lasts)) == 1 else [min(lasts), max(lasts)],
                      "cells_per_run": [min(cells), max(cells)], "ctas": ctas},
           "sequential": {"value": seq_value, "unit": UNIT, "ms_total": ms_seq,
                          "how": "each run its own engine, chunks of dft_stride steps replayed as CUDA graphs"},
           "speedup_vs_sequential": value / seq_value,
           "equal_spectra": {"max_rel_diff_dft": worst, "tolerance": 1e-4},
           "clocks": clk}
    return out


def run_adjoint(args):
    """The inverse-design gradient: the slab device (200 x 200 x 120 cells of 20 nm, CPML 12, FP32, 100 x 100
    x 11 design box of a projected Gaussian random field), 8000 steps, checkpoints every 256 steps. Times the
    forward run (J) and the gradient (recomputation from checkpoints plus the reverse steps) on the device
    clock; the gradient is taken with respect to the design density rho (chain rule through eps). The ratio's
    denominator is a plain forward run of the same engine (the fused pass, no checkpoints); ``forward_ms`` is
    the forward that keeps the checkpoints."""
    import numpy as np
    import torch

    from lightsmith_b200.adjoint import AdjointRun
    from lightsmith_b200.workloads import slab_device_plan

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    plan, box, wE, info = slab_device_plan(n_steps=8000)
    run = AdjointRun(plan, box, wE=wE, checkpoint=256)
    rho = info["rho"]
    eps = info["eps_clad"] + rho[:, :, None] * (info["eps_core"] - info["eps_clad"])
    inv_box = np.broadcast_to(1.0 / eps, tuple(b - a for a, b in box))
    run.set_inv_eps_box(inv_box)
    run.forward(10 * plan["stride"])  # warm-up (kernels, allocator)
    run.backward()
    clocks = Clocks(_gpu_uuid(torch, dev))
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(5)]
    torch.cuda.synchronize(dev)
    ev[3].record()
    run.forward(info["n_steps"], keep=False)  # a plain forward run: no checkpoints
    ev[4].record()
    ev[0].record()
    J, _ = run.forward(info["n_steps"])
    ev[1].record()
    g_inv = run.backward()
    ev[2].record()
    torch.cuda.synchronize(dev)
    clk = clocks.stop()
    t_fwd, t_grad = ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2])
    t_plain = ev[3].elapsed_time(ev[4])
    d_inv = -(info["eps_core"] - info["eps_clad"]) / torch.as_tensor(eps, device=dev) ** 2
    g_rho = (g_inv * d_inv).sum(dim=2)
    cells = int(np.prod(plan["shape"]))
    run.close()
    out = {"metric": "FDTD adjoint gradient time / forward time", "value": t_grad / t_plain, "unit": "ratio",
           "n_gpus": 1, "steps": info["n_steps"], "warmup": 1, "higher_is_better": False, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": "220 nm Si slab in SiO2, 200 x 200 x 120 cells of 20 nm, CPML 12, 2 x 2 um design "
                                  "region (100 x 100 x 11 nodes) of a seeded Gaussian random field (corr. 100 nm, tanh "
                                  "projection beta 8), TE0 slab-mode pulse at 1550 nm, |DFT overlap|^2 on the output "
                                  "plane", "checkpoint_steps": 256},
           "plain_forward_ms": t_plain, "forward_ms": t_fwd, "gradient_ms": t_grad,
           "fused_pass": bool(run.eng.fused),
           "forward_gcells": cells * info["n_steps"] / (t_plain / 1e3) / 1e9,
           "objective": J, "grad_rho_absmax": float(g_rho.abs().max()), "clocks": clk}
    return out


def run_clusters(args):
    """Forward + adjoint over dispersive clusters: ``--instances`` seeded instances of 3-12 silver spheres
    (Drude + 2 Lorentz poles, radii U(10, 40) nm, 2 nm grid). With lightsmith installed each instance is a
    lightsmith ``Simulation`` set up by its own scattering driver (``workloads.cluster_scattering``: its
    table-fed TF/SF plane wave and flux boxes; grids of about 100^3-260^3 cells) and the objective is the sum
    over 24 wavelengths in 350-700 nm of C_sca; without it, a point dipole just outside the shell excites a
    cubic grid sized to the cluster and the objective is the power out of a closed box
    (``workloads.cluster_instance``). The gradient is with respect to the background index of the cells of a
    60 nm shell around the spheres. Each
    instance runs forward (checkpoints every 256 steps) and backward in FP32 on the device clock; the same
    in FP64 gives the errors of each spectrum and each gradient. The instances run one after another (each
    is a whole-GPU grid)."""
    import numpy as np
    import torch

    from lightsmith_b200.adjoint import AdjointRun
    from lightsmith_b200.workloads import cluster_instance, cluster_scattering
    from lightsmith_b200.scattering import cross_section_objective

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    # with lightsmith installed, each instance is posed to it and set up by its own scattering driver (TF/SF
    # plane wave, flux boxes; objective sum_f C_sca); without it, a point dipole and the power out of a box
    posed = _lightsmith_available()
    clocks = Clocks(_gpu_uuid(torch, dev))
    rows, t_f_tot, t_g_tot, cell_steps = [], 0.0, 0.0, 0
    for seed in range(args.instances):
        out = {}
        if posed:  # lightsmith's set-up once per instance; each precision its own objective
            plan, info = cluster_scattering(seed, n_steps=args.cluster_steps)
        for prec in ("single", "double"):
            if posed:
                ref = {}
                info = {**info, "ref": ref, "objective": cross_section_objective(info["post"], ref)}
            else:
                plan, info = cluster_instance(seed, n_steps=args.cluster_steps, single=prec == "single")
            run = AdjointRun(plan, info["box"], objective=info["objective"], checkpoint=256, precision=prec)
            if posed:
                ref["acc_ref"] = run.eng.monitors[2]["acc_e"]
            if prec == "single":  # untimed warm-up of this instance's kernels and graphs
                run.forward(2 * plan["stride"])
                run.backward()
            ev = [torch.cuda.Event(enable_timing=True) for _ in range(3)]
            torch.cuda.synchronize(dev)
            ev[0].record()
            J, (acc_e, acc_h) = run.forward(info["n_steps"])
            ev[1].record()
            g = run.backward()
            ev[2].record()
            torch.cuda.synchronize(dev)
            if posed:
                spectrum = np.asarray(info["ref"]["spectrum"])
            else:
                s = torch.as_tensor(info["sign"], device=acc_e.device)
                spectrum = (0.5 * (acc_e * acc_h.conj() * s).real.sum(dim=1)).cpu().numpy()
            n_bg = info["n_bg"]
            shell = torch.as_tensor(info["shell"], device=g.device)
            g_n = (g * (-2.0 / n_bg ** 3))[shell].cpu().numpy()  # dJ/dn per shell cell (1/eps = 1/n^2)
            out[prec] = (ev[0].elapsed_time(ev[1]), ev[1].elapsed_time(ev[2]), spectrum, g_n, J)
            run.close()
            del run, g, acc_e, acc_h
            torch.cuda.empty_cache()
        tf, tg, s32, g32, J32 = out["single"]
        _, _, s64, g64, J64 = out["double"]
        cells = info["cells"]
        t_f_tot += tf
        t_g_tot += tg
        cell_steps += cells * info["n_steps"]
        rows.append({"seed": seed, "grid": [int(v) for v in plan["shape"]], "spheres": len(info["spheres"]),
                     "shell_cells": int(info["shell"].sum()), "forward_ms": round(tf, 2), "gradient_ms": round(tg, 2),
                     "spectrum_err_vs_fp64": float(np.abs(s32 - s64).max() / max(np.abs(s64).max(), 1e-300)),
                     "gradient_err_vs_fp64": float(np.abs(g32 - g64).max() / max(np.abs(g64).max(), 1e-300))})
    clk = clocks.stop()
    value = cell_steps / ((t_f_tot + t_g_tot) / 1e3) / 1e9
    out = {"metric": "FDTD forward + adjoint gradient over dispersive clusters, Gcell-updates/s of the forward "
                     "steps per second of forward + gradient", "value": value, "unit": UNIT, "n_gpus": 1,
           "steps": args.cluster_steps, "warmup": 1, "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f32", "data": "synthetic",
           "config": {"workload": f"{args.instances} seeded clusters of 3-12 silver spheres (Drude + 2 Lorentz, "
                                  "radii U(10, 40) nm) in n = 1.33, 2 nm grid, CPML 12, " + (
                                      "posed to lightsmith and set up by its scattering driver (table-fed TF/SF "
                                      "plane wave, flux boxes), objective sum_f C_sca at 24 wavelengths in "
                                      "350-700 nm" if posed else "dipole outside the shell, power out of a closed "
                                      "box at 24 wavelengths in 350-700 nm") +
                                  ", gradient in the background index of a 60 nm shell", "checkpoint_steps": 256,
                      "excitation": "TF/SF plane wave (lightsmith's set-up)" if posed else "point dipole"},
           "forward_ms_total": t_f_tot, "gradient_ms_total": t_g_tot, "gradient_over_forward": t_g_tot / t_f_tot,
           "max_spectrum_err_vs_fp64": max(r["spectrum_err_vs_fp64"] for r in rows),
           "max_gradient_err_vs_fp64": max(r["gradient_err_vs_fp64"] for r in rows),
           "instances": rows, "clocks": clk}
    return out


def run_sphere(args):
    """The whole dispersive-sphere scattering solve at full size: the plan lightsmith's scattering driver built
    for an r = 40 nm Drude-Lorentz sphere in n = 1.33 (129^3 cells of 2 nm, CPML 12, table-fed TF/SF, two flux
    boxes and the incident reference view at 81 wavelengths, staircase mesh, dft_stride 100), replayed from
    ``tests/golden/solve_c0.npz`` for its 4000 steps on the CUDA engine in FP32 and FP64. ``value``: Gcell-updates/s
    of the FP32 solve on the device clock (40 chunks replayed as CUDA graphs); ``e2e``: the same solve through
    ``Engine.from_plan`` with the plan's host arrays copied in and the accumulators read back inside the timed
    region. Cross sections (C_ext, C_sca, C_abs at all 81 wavelengths) from the accumulators by the restated
    post-processing, against lightsmith's own engine run on the same plan in FP64, per precision, beside the
    error of lightsmith's own FP32 run of it."""
    import numpy as np
    import torch

    from lightsmith_b200 import plan as P
    from lightsmith_b200.engine import Engine
    from oracle.post import cross_sections

    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    d = P.load(os.path.join(HERE, "tests", "golden", "solve_c0.npz"))
    plan, post, ref = d["plan"], d["post"], d["out"]
    chunks = post["steps"] // plan["stride"]
    cells = int(np.prod(plan["shape"]))
    warm = Engine.from_plan(plan, precision="single")  # untimed: kernels, graphs, allocator
    run, _ = warm.make_runner(True)
    for _ in range(2):
        run()
    warm.close()
    clocks = Clocks(_gpu_uuid(torch, dev))
    # host arrays of the plan (the permittivity, groups, TF/SF tables, monitor and CPML tables), all copied in
    h2d_solve = sum(int(np.asarray(v).nbytes) for v in P.dumps(plan).values())
    res = {}
    for prec in ("single", "double"):
        torch.cuda.synchronize(dev)
        t0 = time.perf_counter()
        eng = Engine.from_plan(plan, precision=prec)
        run, used = eng.make_runner(True)
        ev = [torch.cuda.Event(enable_timing=True) for _ in range(2)]
        ev[0].record(eng.stream)
        for _ in range(chunks):
            run()
        ev[1].record(eng.stream)
        es, hs, d2h = [], [], 0
        for k in range(len(plan["monitors"])):
            e, h = eng.results(k)  # every frequency row, copied to the host
            d2h += np.asarray(e).nbytes + (0 if h is None else np.asarray(h).nbytes)
            es.append(np.asarray(e))
            hs.append(None if h is None else np.asarray(h))
        t1 = time.perf_counter()
        cs = cross_sections(es, hs, post)
        err = {k: float(np.max(np.abs(cs[k] - ref[k]) / np.abs(ref[k]))) for k in ("c_ext", "c_sca", "c_abs")}
        if prec == "single":
            d2h_solve = d2h
            per_wl = {k: (np.abs(cs[k] - ref[k]) / np.abs(ref[k])).tolist() for k in ("c_ext", "c_sca", "c_abs")}
            ls32 = {k: float(np.max(np.abs(ref["lightsmith_fp32"][k] - ref[k]) / np.abs(ref[k])))
                    for k in ("c_ext", "c_sca", "c_abs")}
        res[prec] = {"device_ms": ev[0].elapsed_time(ev[1]), "e2e_ms": (t1 - t0) * 1e3, "err": err,
                     "graphs": bool(used), "fused_pass": bool(getattr(eng, "fused", False))}
        if prec == "single":  # after the solve: the bulk Yee kernels alone, eager, over 4 more chunks
            bulk_ms, bulk_launches = eng.chunk_timed(4)
            res[prec].update(bulk_ms_per_step=bulk_ms / (4 * plan["stride"]), bulk_launches=bulk_launches,
                             launches=eng.launches_per_chunk() * chunks)
        eng.close()
    clk = clocks.stop()
    s = res["single"]
    value = cells * post["steps"] / (s["device_ms"] / 1e3) / 1e9
    from lightsmith_b200.workloads import cells_in_cpml

    alg_bytes = cells * BYTES_PER_CELL + cells_in_cpml(plan) * BYTES_PER_CPML_PAIR
    achieved = alg_bytes / (s["bulk_ms_per_step"] / 1e3) / 1e9
    peak, peak_kind = _peak()
    out = {"metric": "FDTD Gcell-updates/s, whole dispersive-sphere scattering solve", "value": value,
           "unit": UNIT, "n_gpus": 1, "steps": int(post["steps"]), "warmup": 2, "ms_per_step": s["device_ms"] / post["steps"],
           "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
           "data": "lightsmith's own plan for the problem (recorded on the host; no randomness)",
           "config": {"workload": "r = 40 nm Drude-Lorentz sphere (eps_inf 5.9, wp 9 eV, 2 Lorentz poles) in n = 1.33, "
                                  "129^3 cells of 2 nm, CPML 12, table-fed TF/SF plane wave, 81 wavelengths 400-800 nm, "
                                  "staircase, 4000 steps, dft_stride 100", "inputs": "larger than L2 (8.6e6 nodes x 6 "
                                  "fields x 4 B plus CPML and tables)"},
           "e2e": {"value": cells * post["steps"] / (s["e2e_ms"] / 1e3) / 1e9, "unit": UNIT,
                   "h2d_bytes_per_step": h2d_solve // int(post["steps"]),
                   "d2h_bytes_per_step": d2h_solve // int(post["steps"]),
                   "note": "one solve: engine construction from the host plan (its arrays copied in), 4000 steps, "
                           "every accumulator read back; bytes per step are the solve's over its steps"},
           "cross_section_rel_err_vs_lightsmith_fp64": {"fp32": s["err"], "fp64": res["double"]["err"],
                                                        "lightsmith_own_fp32": ls32},
           "fp32_rel_err_per_wavelength": per_wl, "wavelengths_nm": (2 * np.pi / np.asarray(post["omega"])).tolist(),
           "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s", "frac": achieved / peak,
                        "peak_source": peak_kind, "traffic": None,
                        "kernel": "bulk Yee update (H and E with their CPML terms; the in-place kernels on this "
                                  "grid), per FDTD step", "alg_bytes_per_step": alg_bytes,
                        "kernel_ms_per_step": s["bulk_ms_per_step"],
                        "share_of_step": s["bulk_ms_per_step"] / (s["device_ms"] / post["steps"])},
           "fused_pass": s["fused_pass"], "gpu_launches": s["launches"],
           "fp64_solve_ms": res["double"]["device_ms"], "clocks": clk}
    return out


def run_setup(args):
    """Host set-up on the GPU: the meshing of the 129^3 dispersive sphere (the call of lightsmith's ``voxelise``
    that its scattering driver makes, captured from lightsmith's own solve of the problem) by lightsmith on the
    host and by ``lightsmith_b200.voxel`` on the GPU, with the problem's staircase mesh and with subpixel
    smoothing; wall-clock milliseconds (the GPU figure includes its copies and the host assembly, after one
    untimed call), and whether every output is the same bit for bit."""
    import numpy as np
    import torch

    if not _lightsmith_available():
        return {"unavailable": "lightsmith (baseline/_ref) is not installed"}
    sys.path.insert(0, os.path.join(HERE, "tests", "golden"))
    import lightsmith as ls
    from lightsmith.backends._fdtd import scattering as S
    from problems import c0_problem, with_options

    from lightsmith_b200 import voxel

    class Stop(Exception):
        pass

    def captured(prob):
        got = {}
        saved = S._slot_fn, S.voxelise

        def slots(sim, slot_of, n):
            return voxel.ShapeSlots(saved[0](sim, slot_of, n), sim.particles, slot_of)

        def rec(*a, **k):
            got.update(a=a, k=k)
            raise Stop
        S._slot_fn, S.voxelise = slots, rec
        try:
            ls.solve(prob, method="fdtd", device="cpu")
        except Stop:
            pass
        finally:
            S._slot_fn, S.voxelise = saved
        return got["a"], got["k"], saved[1]

    out = {}
    for mode in ("staircase", "subpixel"):
        a, k, host_vox = captured(with_options(c0_problem(), mesh_refinement=mode))
        k = {n: v for n, v in k.items() if n in ("mode", "samples", "base", "background")}
        t0 = time.perf_counter()
        host = host_vox(*a, **k)
        t1 = time.perf_counter()
        voxel.voxelise_gpu(*a, **k, device="cuda:0")  # untimed: library, context and allocator
        torch.cuda.synchronize()
        t2 = time.perf_counter()
        gpu = voxel.voxelise_gpu(*a, **k, device="cuda:0")
        t3 = time.perf_counter()
        same = bool(np.array_equal(host[0], gpu[0]) and host[2] == gpu[2] and len(host[1]) == len(gpu[1]) and all(
            np.array_equal(g.idx, h.idx) and np.array_equal(g.frac, h.frac) for g, h in zip(gpu[1], host[1])))
        out[mode] = {"host_ms": (t1 - t0) * 1e3, "gpu_ms": (t3 - t2) * 1e3, "speedup": (t1 - t0) / max(t3 - t2, 1e-9),
                     "interface_cells": int(host[2]["interface_cells"]), "identical": same}
    return {"workload": "meshing of the 129^3 Drude-Lorentz sphere (r = 40 nm, 2 nm cells) as lightsmith's "
                        "scattering driver calls voxelise", **out}


def forms(args) -> dict:
    """The method's other forms on this GPU, each a record with its own clock samples, for the default line:
    the whole 129^3 dispersive-sphere solve (Gcell/s, roofline of its bulk kernel, FP32 and FP64 errors), the
    batched oblique sweep against the same runs one after another, the adjoint gradient's cost over a forward
    run, forward + gradient over dispersive clusters with FP64 errors (a few instances), and the sphere's host
    set-up (meshing) on the host and on the GPU."""
    import torch

    out = {}
    for name, fn, kw in (("sphere", run_sphere, {}), ("sweep", run_sweep, {}), ("adjoint", run_adjoint, {}),
                         ("clusters", run_clusters, {"instances": args.form_instances}), ("setup", run_setup, {})):
        sub = argparse.Namespace(**{**vars(args), **kw})
        t0 = time.perf_counter()
        try:
            rec = fn(sub)
        except Exception as e:  # noqa: BLE001 (one form failing must not lose the headline line)
            rec = {"error": f"{type(e).__name__}: {e}"}
        rec["wall_s"] = round(time.perf_counter() - t0, 2)
        out[name] = rec
        torch.cuda.empty_cache()
    return out


def main():
    args = _args()
    if args.impl == "reference":
        run_reference(args)
    elif args.workload == "sweep":
        print(json.dumps(run_sweep(args)), flush=True)
    elif args.workload == "adjoint":
        print(json.dumps(run_adjoint(args)), flush=True)
    elif args.workload == "clusters":
        print(json.dumps(run_clusters(args)), flush=True)
    elif args.workload == "sphere":
        print(json.dumps(run_sphere(args)), flush=True)
    elif args.workload == "setup":
        print(json.dumps(run_setup(args)), flush=True)
    else:
        run_b200(args)


if __name__ == "__main__":
    main()

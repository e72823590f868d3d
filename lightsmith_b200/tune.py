"""Launch-shape tuning of the fused FDTD step, and a fixed-shape run for profiling.

The fused single pass has three knobs: CTA tile rows along y (8 or 16), x planes per CTA, and the depth of
its copy ring. ``tune_engine`` times each candidate on an engine with CUDA events around the bulk kernel
(eager chunks, so the fields keep evolving; the kernel's time does not depend on their values) and leaves
the engine on the fastest. ``best_shape`` caches the choice per GPU model and grid shape in a JSON file.

    python -m lightsmith_b200.tune --n 640                  # sweep the throughput case, print the best
    python -m lightsmith_b200.tune --n 384 --shape 3,8,32,4   # one shape (e.g. under ncu)
    python -m lightsmith_b200.tune --plan run.npz --shape 4,8,0,4  # a recorded plan (lightsmith_b200.plan.save)
"""

from __future__ import annotations

import argparse
import json
import os

# (variant, tile rows, x planes per tile, ring depth): variant 0 the in-place kernels, 2 their four-node
# vector form, 1 the fused pass, 3 the fused pass split into an interior box and the CPML/wall shell, 4 the
# fused pass with lean CPML terms; planes 0 lets the engine choose per grid (48, fewer on small grids)
CANDIDATES = [(0, 8, 32, 4), (2, 8, 32, 4), (1, 8, 0, 4), (1, 16, 0, 4), (3, 8, 0, 4), (3, 16, 0, 4),
              (4, 8, 0, 4), (4, 16, 0, 4), (4, 8, 8, 4), (4, 8, 24, 4), (4, 8, 48, 4), (4, 8, 64, 4)]


def _cache_path() -> str:
    base = os.environ.get("XDG_CACHE_HOME", os.path.join(os.path.expanduser("~"), ".cache"))
    return os.path.join(base, "lightsmith_b200", "tuning.json")


def time_shape(eng, shape, chunks: int = 2) -> float:
    """Milliseconds of bulk-kernel time per FDTD step under launch shape (variant, tile_y, planes, stages)."""
    eng.set_tuning(*shape)
    eng.chunk_timed(1)  # first launch of a shape pays its set-up
    ms, _ = eng.chunk_timed(chunks)
    eng.check_status()
    return ms / (chunks * eng.stride)


def tune_engine(eng, candidates=CANDIDATES, chunks: int = 2):
    """Time every candidate (eager chunks, before any graph capture); leave the engine on the fastest.
    Returns (best shape, {shape: ms per step})."""
    res = {tuple(c): time_shape(eng, c, chunks) for c in candidates}
    best = min(res, key=res.get)
    eng.set_tuning(*best)
    return best, res


def best_shape(eng, candidates=CANDIDATES, path: str | None = None):
    """The cached best shape for this GPU model and grid shape, tuning (and caching) it on a miss."""
    import torch

    import zlib

    cands = zlib.crc32(repr([tuple(c) for c in candidates]).encode())  # a new candidate list tunes afresh
    key = (f"{torch.cuda.get_device_name(eng.dev)}|{'x'.join(map(str, eng.shape))}|"
           f"{'f32' if eng.single else 'f64'}|{cands:08x}")
    path = path or _cache_path()
    cache = {}
    try:
        with open(path) as f:
            cache = json.load(f)
    except (OSError, ValueError):
        pass
    if key in cache:
        shape = tuple(cache[key])
        eng.set_tuning(*shape)
        return shape
    best, _ = tune_engine(eng, candidates)
    if best is not None:
        cache[key] = list(best)
        try:
            os.makedirs(os.path.dirname(path), exist_ok=True)
            with open(path, "w") as f:
                json.dump(cache, f, indent=1)
        except OSError:
            pass
    return best


# (CTAs per run, runs in flight; 0: as many as fit): clusters of 4, 8 or 16 CTAs, groups of 37 or 74 CTAs, and
# the default (0: groups of half the resident CTAs)
BATCH_SHAPES = [(0, 0), (8, 0), (4, 0), (16, 0), (37, 0), (74, 0)]


def tune_batch(engines, last, shapes=BATCH_SHAPES, steps: int = 30, launches: int = 2):
    """Time the batched kernel's launch shapes on ``engines`` (which advance: tune on runs made for it) and
    return (best shape, {shape: Gcell-updates/s})."""
    import numpy as np
    import torch

    from .batch import BlochBatch

    cells = [int(np.prod(e.shape)) for e in engines]
    res = {}
    for cl, mx in shapes:
        try:
            b = BlochBatch(engines, last, cluster_ctas=cl, max_clusters=mx)
        except Exception:  # noqa: BLE001 (a shape the device cannot launch)
            continue
        b.run(steps, 1)  # capture
        t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        before = [e.n_host for e in engines]
        t0.record(b.stream)
        b.run(steps, launches)
        t1.record(b.stream)
        torch.cuda.synchronize()
        moved = sum(c * (e.n_host - n) for c, e, n in zip(cells, engines, before))
        res[(cl, mx)] = moved / max(t0.elapsed_time(t1), 1e-9) / 1e6
        b.close()
    best = max(res, key=res.get) if res else (0, 0)
    return best, res


# steps a run advances per visit of its CTAs (one launch): while in flight a run's fields stay in L2 from one
# step to the next, and the steps of a visit reuse them; fewer steps switch runs (and reload them) more often
BATCH_DEPTHS = (8, 32, 128, 512)


def tune_batch_depth(engines, last, shape=(0, 0), depths=BATCH_DEPTHS, launches: int = 2):
    """Time the batched kernel's steps per visit (the depth of its L2-resident blocking in time) under launch
    shape ``shape`` on ``engines`` (which advance) and return (best depth, {depth: Gcell-updates/s})."""
    import numpy as np
    import torch

    from .batch import BlochBatch

    cells = [int(np.prod(e.shape)) for e in engines]
    res = {}
    b = BlochBatch(engines, last, cluster_ctas=shape[0], max_clusters=shape[1])
    try:
        for depth in depths:
            b.run(depth, 1)  # capture the graph of this step count
            t0, t1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            before = [e.n_host for e in engines]
            t0.record(b.stream)
            b.run(depth, launches)
            t1.record(b.stream)
            torch.cuda.synchronize()
            moved = sum(c * (e.n_host - n) for c, e, n in zip(cells, engines, before))
            if moved:
                res[int(depth)] = moved / max(t0.elapsed_time(t1), 1e-9) / 1e6
    finally:
        b.close()
    best = max(res, key=res.get) if res else int(depths[-1])
    return best, res


def _main():
    import torch

    from .engine import Engine
    from .workloads import cells_in_cpml, throughput_plan

    ap = argparse.ArgumentParser()
    ap.add_argument("--n", type=int, default=384)
    ap.add_argument("--shape", default=None, help="variant,tile_y,planes,stages: time only this launch shape")
    ap.add_argument("--chunks", type=int, default=2)
    ap.add_argument("--cp-async", action="store_true", help="copy planes with cp.async instead of TMA")
    ap.add_argument("--pml", type=int, default=16, help="CPML cells on every face")
    ap.add_argument("--plan", default=None, help="a plan saved with lightsmith_b200.plan.save, run in FP32")
    ap.add_argument("--whole", action="store_true",
                    help="variant 4: step every tile with the lean kernel (no clean-interior kernel)")
    args = ap.parse_args()
    if args.plan:
        from .plan import load

        d = load(args.plan)
        plan = d.get("plan", d)
        eng = Engine.from_plan(plan, precision="single")
    else:
        n = args.n
        inv = 1.0 / (torch.rand((n, n, n), device="cuda", dtype=torch.float32) * 11.25 + 1.0)
        plan = throughput_plan(n, inv_eps=inv, max_steps=31 * 200, pml=args.pml)
        del inv
        eng = Engine.from_plan(plan)
    if args.cp_async:
        eng.set_copy_engine(False)
    if args.whole:
        eng.set_clean_split(False)
    cells = eng.cells
    alg = cells * 52 + cells_in_cpml(eng.plan) * 32
    shapes = [tuple(int(v) for v in args.shape.split(","))] if args.shape else CANDIDATES
    for sh in shapes:
        ms = time_shape(eng, sh, args.chunks)
        print(json.dumps({"shape": sh, "fused": eng.fused, "tma": eng.uses_tma, "whole": args.whole, "ms_per_step": ms,
                          "Gcell_s": cells / ms / 1e6, "alg_GBps": alg / ms / 1e6}), flush=True)
    eng.close()


if __name__ == "__main__":
    _main()

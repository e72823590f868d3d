"""Launch-shape tuning of the fused FDTD step, and a fixed-shape run for profiling.

The fused single pass has three knobs: CTA tile rows along y (8 or 16), x planes per CTA, and the depth of
its copy ring. ``tune_engine`` times each candidate on an engine with CUDA events around the bulk kernel
(eager chunks, so the fields keep evolving; the kernel's time does not depend on their values) and leaves
the engine on the fastest. ``best_shape`` caches the choice per GPU model and grid shape in a JSON file.

    python -m lightsmith_b200.tune --n 640                  # sweep the throughput case, print the best
    python -m lightsmith_b200.tune --n 384 --shape 3,8,32,4   # one shape (e.g. under ncu)
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
    args = ap.parse_args()
    n = args.n
    inv = 1.0 / (torch.rand((n, n, n), device="cuda", dtype=torch.float32) * 11.25 + 1.0)
    plan = throughput_plan(n, inv_eps=inv, max_steps=31 * 200, pml=args.pml)
    del inv
    eng = Engine.from_plan(plan)
    if args.cp_async:
        eng.set_copy_engine(False)
    alg = n ** 3 * 52 + cells_in_cpml(eng.plan) * 32
    shapes = [tuple(int(v) for v in args.shape.split(","))] if args.shape else CANDIDATES
    for sh in shapes:
        ms = time_shape(eng, sh, args.chunks)
        print(json.dumps({"shape": sh, "tma": eng.uses_tma, "ms_per_step": ms, "Gcell_s": n ** 3 / ms / 1e6,
                          "alg_GBps": alg / ms / 1e6}), flush=True)
    eng.close()


if __name__ == "__main__":
    _main()

"""Autotuner: picks launch shapes and the brick size by timing the candidates
on the caller's own data with CUDA events (no reference counterpart).

  tune_query_batch  threads per CTA and tile run length of the batched query launch
                    (128 / 256 / 512), set on the QueryBatch;
  tune_block_dim    sparse brick edge (4 / 8 / 16 voxels) for a mesh and a
                    query set: builds each candidate grid and times its
                    queries -- smaller bricks store fewer voxels outside the
                    band, larger ones need fewer table lookups per query;
  tune_fill_ctas    CTAs per SM of the persistent batched brick fill.

  tune_fill_tile    voxel tile of the dense fill CTAs (8x8x4, 4x4x16, ...):
                    the warp's voxel patch sets how coherent its traversals
                    are; every shape builds the same grid bit for bit;
  tune_host_chunk   queries per pipelined chunk of sdfo_query_host.

Results are plain dicts so they can be stored next to a workload and
re-applied without re-timing; ``TuningCache`` keeps them in a JSON file keyed
by (GPU name, workload shape) and applies stored knobs through
sdfo_set_tuning.
"""
from __future__ import annotations

import json
import os

from . import _native as N


def _time(fn, reps, warmup):
    import torch

    for _ in range(warmup):
        fn()
    stream = torch.cuda.current_stream()
    start = torch.cuda.Event(enable_timing=True)
    stop = torch.cuda.Event(enable_timing=True)
    start.record(stream)
    for _ in range(reps):
        fn()
    stop.record(stream)
    stop.synchronize()
    return start.elapsed_time(stop) / reps


def tune_query_batch(batch, points, poses=None, mode=N.TRICUBIC, candidates=(128, 256, 512),
                     runs=(1, 2, 4, 8), reps=20, warmup=3):
    """Times QueryBatch.run for each CTA size and tile run length, keeps the
    fastest on the batch; returns {"threads": t, "run": r, "ms":
    {"<t>x<r>": ms}}."""
    out = batch.outputs(points.device)
    ms = {}
    for t in candidates:
        batch.set_threads(t)
        for r in runs:
            batch.set_run(r)
            ms[(t, r)] = _time(lambda: batch.run(points, poses, mode, out), reps, warmup)
    best = min(ms, key=ms.get)
    batch.set_threads(best[0])
    batch.set_run(best[1])
    return {"threads": best[0], "run": best[1], "ms": {f"{t}x{r}": v for (t, r), v in ms.items()}}


def tune_block_dim(verts, tris, points, candidates=(4, 8, 16), mode=N.TRICUBIC, reps=20,
                   warmup=3, **build_kwargs):
    """Builds the sparse grid with each brick edge and times the Tricubic
    query of ``points`` (CUDA float32 (N,3)); returns {"block_dim": best,
    "ms": {...}, "stored_voxels": {...}}.  Only candidates whose grids keep
    every point's validity are eligible (a larger brick never loses
    coverage; a smaller one can only add invalid points)."""
    from .grid import SdfGrid

    ms, stored, valid = {}, {}, {}
    for bd in candidates:
        g = SdfGrid.build_sparse(verts, tris, block_dim=bd, mode=mode, **build_kwargs)
        out = g.query_tensors(points, mode=mode, valid=True)
        valid[bd] = int(out["valid"].sum().item())
        ms[bd] = _time(lambda: g.query_tensors(points, mode=mode, valid=True), reps, warmup)
        stored[bd] = g.stored_voxels
        g.close()
    most = max(valid.values())
    eligible = [bd for bd in candidates if valid[bd] == most]
    best = min(eligible, key=lambda bd: ms[bd])
    return {"block_dim": best, "ms": ms, "stored_voxels": stored, "valid": valid}


def tune_fill_ctas(meshes, candidates=(1, 2, 4), reps=1):
    """Times the batched sparse build with the persistent fill limited to
    ``k`` CTAs per SM; returns {"ctas_per_sm": best, "ms": {...}} and leaves
    the best setting active (process-wide, sdfo_set_fill_ctas_per_sm)."""
    from .grid import SdfGrid

    lib = N.load()
    ms = {}
    for k in candidates:
        N.check(lib.sdfo_set_fill_ctas_per_sm(int(k)))
        total = 0.0
        for _ in range(reps):
            grids = SdfGrid.build_sparse_batched(meshes)
            total += grids[0].build_stats()["fill_ms"]
            for g in grids:
                g.close()
        ms[k] = total / reps
    best = min(ms, key=ms.get)
    N.check(lib.sdfo_set_fill_ctas_per_sm(int(best)))
    return {"ctas_per_sm": best, "ms": ms}


def tune_fill_tile(verts, tris, candidates=((3, 3), (2, 2), (3, 2), (4, 2), (2, 3), (4, 1)), reps=2,
                   **build_kwargs):
    """Times the dense build's fill with each voxel tile (log2 x, log2 y)
    and leaves the fastest set (process-wide); returns {"tile": best,
    "fill_ms": {...}}."""
    from .grid import SdfGrid

    ms = {}
    for lx, ly in candidates:
        N.set_tuning(fill_tile_log2_x=lx, fill_tile_log2_y=ly)
        SdfGrid.build_dense(verts, tris, **build_kwargs).close()  # warm
        total = 0.0
        for _ in range(reps):
            g = SdfGrid.build_dense(verts, tris, **build_kwargs)
            total += g.build_stats()["fill_ms"]
            g.close()
        ms[(lx, ly)] = total / reps
    best = min(ms, key=ms.get)
    N.set_tuning(fill_tile_log2_x=best[0], fill_tile_log2_y=best[1])
    return {"tile": best, "fill_ms": {f"{k[0]},{k[1]}": v for k, v in ms.items()}}


def tune_host_chunk(grid, points, mode=N.TRICUBIC, candidates=(65536, 131072, 262144, 524288, 1 << 30),
                    reps=20, warmup=3):
    """Times sdfo_query_host on ``points`` (a pinned float32 (N,3) CPU
    tensor) with each chunk size and leaves the fastest set; returns
    {"host_chunk_queries": best, "ms": {...}}."""
    import ctypes
    import time

    import torch

    n = points.shape[0]
    gap = torch.empty(n).pin_memory()
    grad = torch.empty((n, 3)).pin_memory()
    valid = torch.empty(n, dtype=torch.uint8).pin_memory()
    P = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    lib = N.load()

    def call():
        N.check(lib.sdfo_query_host(grid.handle, mode, P(points), 0, n, P(gap), P(grad), None, None,
                                    P(valid), None))

    ms = {}
    for c in candidates:
        N.set_tuning(host_chunk_queries=int(min(c, 1 << 30)))
        for _ in range(warmup):
            call()
        t0 = time.perf_counter()
        for _ in range(reps):
            call()
        ms[int(c)] = 1e3 * (time.perf_counter() - t0) / reps
    best = min(ms, key=ms.get)
    N.set_tuning(host_chunk_queries=best)
    return {"host_chunk_queries": best, "ms": ms}


def gpu_name(device=0) -> str:
    import torch

    return torch.cuda.get_device_name(device)


class TuningCache:
    """Tuned knobs in a JSON file: {"<gpu name>|<workload key>": {knob: value}}.
    The default file is $SDFO_TUNING_CACHE, else ~/.cache/sdfo/tuning.json."""

    def __init__(self, path=None):
        self.path = path or os.environ.get("SDFO_TUNING_CACHE") or os.path.join(
            os.path.expanduser("~"), ".cache", "sdfo", "tuning.json")
        self.data = {}
        if os.path.exists(self.path):
            with open(self.path) as f:
                self.data = json.load(f)

    @staticmethod
    def key(gpu: str, workload: str) -> str:
        return f"{gpu}|{workload}"

    def get(self, gpu: str, workload: str):
        return self.data.get(self.key(gpu, workload))

    def put(self, gpu: str, workload: str, knobs: dict) -> None:
        self.data[self.key(gpu, workload)] = dict(knobs)
        os.makedirs(os.path.dirname(os.path.abspath(self.path)), exist_ok=True)
        tmp = self.path + ".tmp"
        with open(tmp, "w") as f:
            json.dump(self.data, f, indent=1, sort_keys=True)
        os.replace(tmp, self.path)

    def apply(self, gpu: str, workload: str) -> bool:
        """Sets the stored sdfo_set_tuning knobs of (gpu, workload); returns
        whether an entry existed.  Knobs that are not sdfo_tuning fields
        (e.g. a QueryBatch's threads) are left to the caller."""
        knobs = self.get(gpu, workload)
        if knobs is None:
            return False
        fields = {name for name, _ in N.Tuning._fields_}
        N.set_tuning(**{k: v for k, v in knobs.items() if k in fields})
        return True

    def apply_batch(self, gpu: str, workload: str, batch) -> bool:
        """Sets a stored launch shape ("threads", "run": what
        tune_query_batch picks) on a QueryBatch; returns whether the entry
        held one."""
        knobs = self.get(gpu, workload) or {}
        if "threads" not in knobs and "run" not in knobs:
            return False
        if "threads" in knobs:
            batch.set_threads(int(knobs["threads"]))
        if "run" in knobs:
            batch.set_run(int(knobs["run"]))
        return True


def workload_key(kind: str, shape, **extra) -> str:
    """A stable key for a workload shape, e.g. workload_key("dense_fill",
    (128, 128, 64), tris=34816)."""
    parts = [kind, "x".join(str(int(v)) for v in shape)]
    parts += [f"{k}={extra[k]}" for k in sorted(extra)]
    return ":".join(parts)


__all__ = ["tune_query_batch", "tune_block_dim", "tune_fill_ctas", "tune_fill_tile", "tune_host_chunk",
           "TuningCache", "workload_key", "gpu_name"]

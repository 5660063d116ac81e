"""Autotuner: picks launch shapes and the brick size by timing the candidates
on the caller's own data with CUDA events (no reference counterpart).

  tune_query_batch  threads per CTA of the batched query launch
                    (128 / 256 / 512), set on the QueryBatch;
  tune_block_dim    sparse brick edge (4 / 8 / 16 voxels) for a mesh and a
                    query set: builds each candidate grid and times its
                    queries -- smaller bricks store fewer voxels outside the
                    band, larger ones need fewer table lookups per query;
  tune_fill_ctas    CTAs per SM of the persistent batched brick fill.

Results are plain dicts so they can be stored next to a workload and
re-applied without re-timing.
"""
from __future__ import annotations

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
                     reps=20, warmup=3):
    """Times QueryBatch.run for each CTA size, keeps the fastest on the batch;
    returns {"threads": best, "ms": {threads: ms}}."""
    out = batch.outputs(points.device)
    ms = {}
    for t in candidates:
        batch.set_threads(t)
        ms[t] = _time(lambda: batch.run(points, poses, mode, out), reps, warmup)
    best = min(ms, key=ms.get)
    batch.set_threads(best)
    return {"threads": best, "ms": ms}


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


__all__ = ["tune_query_batch", "tune_block_dim", "tune_fill_ctas"]

"""Many grids at once: the batched sparse build and the one-launch query over
many grids under rigid poses (sdfo_grid_build_sparse_batched,
sdfo_query_batch_*), plus CUDA-graph capture of the batched query.

No reference counterpart: the reference builds and queries one SdfOracle at
a time (SdfBuilder::buildSparse, SdfOracle::queryBatch).
"""
from __future__ import annotations

import ctypes

import numpy as np

from . import _native as N
from .grid import SdfGrid, _stream_ptr, _t_ptr


def build_sparse_batched(meshes, mode=N.TRICUBIC, stream=None):
    """One SdfGrid per mesh dict (verts, tris, build_sparse keywords)."""
    return SdfGrid.build_sparse_batched(meshes, mode=mode, stream=stream)


def pack_poses(R, t, device="cuda"):
    """(n,3,3) rotations (grid to world) and (n,3) translations -> the device
    array of sdfo_pose records, as a (n, 12) float64 tensor."""
    import torch

    R = np.asarray(R, np.float64).reshape(-1, 9)
    t = np.asarray(t, np.float64).reshape(-1, 3)
    return torch.tensor(np.concatenate([R, t], axis=1), dtype=torch.float64, device=device)


class QueryBatch:
    """Queries of ``counts[g]`` consecutive points on grid ``g``, for all grids
    in one launch.  The grids must stay alive while the batch is used (the
    batch keeps a reference)."""

    def __init__(self, grids, counts):
        self._lib = N.load()
        self.grids = list(grids)
        n = len(self.grids)
        self.counts = np.ascontiguousarray(counts, np.int64)
        if self.counts.shape != (n,):
            raise ValueError("one count per grid")
        arr = (ctypes.c_void_p * n)(*[g.handle for g in self.grids])
        out = ctypes.c_void_p()
        N.check(self._lib.sdfo_query_batch_create(arr, n, ctypes.c_void_p(self.counts.ctypes.data),
                                                  ctypes.byref(out)))
        self.handle = out.value
        self.total = int(self.counts.sum())
        self.threads = 128
        self.run_tiles = 4

    def set_threads(self, threads: int) -> None:
        N.check(self._lib.sdfo_query_batch_set_threads(self.handle, int(threads)))
        self.threads = int(threads)

    def set_run(self, tiles: int) -> None:
        """Consecutive tiles each persistent CTA takes before it strides
        (a power of two, 1..64)."""
        N.check(self._lib.sdfo_query_batch_set_run(self.handle, int(tiles)))
        self.run_tiles = int(tiles)

    def outputs(self, device="cuda"):
        """Preallocated (gap, grad, valid) for run(..., out=...), e.g. for a
        CUDA graph."""
        import torch

        return (torch.empty(self.total, dtype=torch.float32, device=device),
                torch.empty((self.total, 3), dtype=torch.float32, device=device),
                torch.empty(self.total, dtype=torch.uint8, device=device))

    def run(self, points, poses=None, mode=N.TRICUBIC, out=None, stream=None):
        """points (total, 3) float32 CUDA tensor (world frame); poses (n, 12)
        float64 CUDA tensor from pack_poses or None -> (gap, grad, valid)."""
        import torch

        if points.dtype != torch.float32 or not points.is_cuda or not points.is_contiguous():
            raise ValueError("points must be a contiguous CUDA float32 tensor")
        if points.shape != (self.total, 3):
            raise ValueError(f"points must have shape ({self.total}, 3)")
        if poses is not None and (poses.dtype != torch.float64 or
                                  tuple(poses.shape) != (len(self.grids), 12)):
            raise ValueError("poses must be a (n, 12) float64 tensor (pack_poses)")
        gap, grad, valid = out if out is not None else self.outputs(points.device)
        N.check(self._lib.sdfo_query_batch_run(self.handle, N.mode_id(mode), _t_ptr(points),
                                               _t_ptr(poses), _t_ptr(gap), _t_ptr(grad),
                                               _t_ptr(valid), _stream_ptr(stream)))
        return gap, grad, valid

    def capture(self, points, poses=None, mode=N.TRICUBIC, out=None):
        """A torch.cuda.CUDAGraph replaying run() on these tensors, and its
        output tensors."""
        import torch

        out = out if out is not None else self.outputs(points.device)
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            self.run(points, poses, mode, out, stream=side)  # warm-up outside the capture
        torch.cuda.current_stream().wait_stream(side)
        graph = torch.cuda.CUDAGraph()
        with torch.cuda.graph(graph):
            self.run(points, poses, mode, out)
        return graph, out

    def close(self) -> None:
        if getattr(self, "handle", None):
            self._lib.sdfo_query_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

"""SdfGrid: a device-resident SDF grid behind the libsdfo_cuda C ABI.

Mirrors the reference's two front ends:

* the C++ SdfBuilder / SdfOracle API (plugins/SdfOracle/include/SdfOracle/
  SdfBuilder.h:58-113, SdfOracle.h:20-67): ``SdfGrid.build_dense``,
  ``SdfGrid.build_sparse``, ``query`` with the five QueryMode values, the
  GridSpec fields and ``load`` / ``save`` of the SDFO 0.1.0 file;
* the Python grid duck type used by SDFContactEngine
  (prototype/src/sdf_grid.py:25-204): ``query(y)`` and ``query_batch(Y)``
  returning ``(g, raw_grad, grad_norm, unit_normal, valid)`` and the
  attributes ``bmin``, ``bmax``, ``voxel``, ``nx``, ``ny``, ``nz``.

Everything runs on the GPU; there is no CPU fallback.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

from . import _native as N


def _torch():
    import torch

    return torch


def _stream_ptr(stream=None):
    torch = _torch()
    s = stream if stream is not None else torch.cuda.current_stream()
    return ctypes.c_void_p(s.cuda_stream)


def _np_ptr(a):
    return None if a is None else ctypes.c_void_p(a.ctypes.data)


def _t_ptr(t):
    return None if t is None else ctypes.c_void_p(t.data_ptr())


class SdfGrid:
    """Owning handle to a device grid (dense or sparse narrow band)."""

    def __init__(self, handle: int, mode=N.TRILINEAR, _keepalive=None):
        if not handle:
            raise ValueError("null grid handle")
        self._h = ctypes.c_void_p(handle)
        self._lib = N.load()
        self._keepalive = _keepalive
        self.mode = N.mode_id(mode)
        self._refresh_info()

    # ------------------------------------------------------------------ life
    def close(self) -> None:
        if getattr(self, "_h", None) and self._h.value:
            self._lib.sdfo_grid_destroy(self._h)
            self._h = ctypes.c_void_p(None)

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def handle(self) -> ctypes.c_void_p:
        if not self._h.value:
            raise RuntimeError("grid is closed")
        return self._h

    def _refresh_info(self) -> None:
        info = N.GridInfo()
        N.check(self._lib.sdfo_grid_get_info(self._h, ctypes.byref(info)))
        self.info = info
        self.bmin = np.array(info.bmin[:], dtype=np.float64)
        self.bmax = np.array(info.bmax[:], dtype=np.float64)
        self.voxel = np.array(info.voxel[:], dtype=np.float64)
        self.shape = tuple(int(x) for x in info.shape)
        self.nx, self.ny, self.nz = self.shape
        self.is_sparse = info.layout == N.LAYOUT_SPARSE
        self.has_hessian = bool(info.has_hessian)
        self.block_dim = int(info.block_dim)
        self.halo_voxels = int(info.halo_voxels)
        self.block_count = int(info.block_count)
        self.band_distance = float(info.band_distance)
        self.storage = int(info.storage)
        self.candidate_stride = int(info.candidate_stride)
        views = N.DeviceViews()
        N.check(self._lib.sdfo_grid_device_views(self._h, ctypes.byref(views)))
        self.stored_voxels = int(views.stored_voxels)

    def spec(self) -> dict:
        return dict(bmin=self.bmin.copy(), bmax=self.bmax.copy(), voxel=self.voxel.copy(),
                    shape=self.shape)

    # --------------------------------------------------------------- builds
    @staticmethod
    def _mesh(verts, tris):
        v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
        t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 3)
        return v, t

    @classmethod
    def build_dense(cls, verts, tris, padding=0.1, voxel_size=0.0, target_resolution=128,
                    max_resolution=512, mode=N.TRILINEAR, stream=None) -> "SdfGrid":
        """SdfBuilder::build (SdfBuilder.cpp:364-407) on the GPU."""
        v, t = cls._mesh(verts, tris)
        lib = N.load()
        p = N.BuildParams(padding, voxel_size, target_resolution, max_resolution)
        out = ctypes.c_void_p()
        N.check(lib.sdfo_grid_build_dense(_np_ptr(v), len(v), _np_ptr(t), len(t), ctypes.byref(p),
                                          _stream_ptr(stream), ctypes.byref(out)))
        return cls(out.value, mode)

    @classmethod
    def traversal_stats(cls, verts, tris, padding=0.1, voxel_size=0.0, target_resolution=128,
                        max_resolution=512, stream=None) -> dict:
        """Per-voxel traversal work of build_dense's fill on the same grid
        (nearest search: nodes examined, closest-point tests; parity ray:
        box tests, triangle tests), counted on the device."""
        v, t = cls._mesh(verts, tris)
        p = N.BuildParams(padding, voxel_size, target_resolution, max_resolution)
        st = N.TraversalStats()
        N.check(N.load().sdfo_build_traversal_stats(_np_ptr(v), len(v), _np_ptr(t), len(t),
                                                    ctypes.byref(p), _stream_ptr(stream),
                                                    ctypes.byref(st)))
        n = max(st.voxels, 1)
        return {"voxels": st.voxels,
                "totals": [st.nearest_nodes, st.nearest_triangles, st.ray_nodes, st.ray_triangles],
                "nearest_nodes_per_voxel": st.nearest_nodes / n,
                "nearest_triangle_tests_per_voxel": st.nearest_triangles / n,
                "ray_box_tests_per_voxel": st.ray_nodes / n,
                "ray_triangle_tests_per_voxel": st.ray_triangles / n,
                "exact_triangle_tests_per_voxel": st.nearest_triangles_exact / n}

    @classmethod
    def build_sparse(cls, verts, tris, padding=0.1, voxel_size=0.0, target_resolution=128,
                     max_resolution=512, block_dim=8, halo_voxels=2, band_voxels=8,
                     band_distance=0.0, store_hessian=True, mode=N.TRILINEAR,
                     stream=None) -> "SdfGrid":
        """SdfBuilder::buildSparse (SdfBuilder.cpp:823-983) on the GPU."""
        v, t = cls._mesh(verts, tris)
        lib = N.load()
        p = N.SparseBuildParams(N.BuildParams(padding, voxel_size, target_resolution,
                                              max_resolution),
                                block_dim, halo_voxels, band_voxels, 1 if store_hessian else 0,
                                band_distance)
        out = ctypes.c_void_p()
        N.check(lib.sdfo_grid_build_sparse(_np_ptr(v), len(v), _np_ptr(t), len(t),
                                           ctypes.byref(p), _stream_ptr(stream),
                                           ctypes.byref(out)))
        return cls(out.value, mode)

    @classmethod
    def build_contact_aware(cls, verts, tris, corner_normals, padding=0.1, voxel_size=0.0,
                            target_resolution=128, max_resolution=512, max_candidates=4,
                            feature_distance_tolerance=0.0, normal_merge_angle_degrees=5.0,
                            tile_dim=8, use_tile_acceleration=True, store_hessian=True,
                            sparse=False, block_dim=8, halo_voxels=2, band_voxels=8,
                            band_distance=0.0, mode=N.CONTACT_AWARE, stream=None) -> "SdfGrid":
        """SdfBuilder::buildContactAware / buildSparseContactAware
        (SdfBuilder.cpp:416-821) on the GPU; corner_normals (nt, 3, 3)."""
        v, t = cls._mesh(verts, tris)
        cn = np.ascontiguousarray(corner_normals, np.float64).reshape(-1, 3, 3)
        if len(cn) != len(t):
            raise ValueError("one corner-normal triplet per triangle is required")
        lib = N.load()
        p = N.ContactAwareParams()
        lib.sdfo_contact_aware_params_default(ctypes.byref(p))
        p.base = N.BuildParams(padding, voxel_size, target_resolution, max_resolution)
        p.max_candidates = max_candidates
        p.tile_dim = tile_dim
        p.use_tile_acceleration = 1 if use_tile_acceleration else 0
        p.store_hessian = 1 if store_hessian else 0
        p.feature_distance_tolerance = feature_distance_tolerance
        p.normal_merge_angle_degrees = normal_merge_angle_degrees
        p.sparse = 1 if sparse else 0
        p.block_dim = block_dim
        p.halo_voxels = halo_voxels
        p.band_voxels = band_voxels
        p.band_distance = band_distance
        out = ctypes.c_void_p()
        N.check(lib.sdfo_grid_build_contact_aware(_np_ptr(v), len(v), _np_ptr(t), len(t),
                                                  _np_ptr(cn), ctypes.byref(p), _stream_ptr(stream),
                                                  ctypes.byref(out)))
        return cls(out.value, mode)

    def export_candidates(self) -> dict:
        """Contact-aware candidates in stored-voxel order: stride, count (N,),
        phi (N,s), normal (N,s,3), branch (N,s) (sparse: FP32 values)."""
        s = self.candidate_stride
        if s <= 0:
            raise ValueError("grid has no contact-aware candidates")
        n = self.stored_voxels
        out = dict(stride=s, count=np.zeros(n, np.uint8), phi=np.zeros((n, s)),
                   normal=np.zeros((n, s, 3)), branch=np.zeros((n, s), np.int32))
        _torch().cuda.synchronize()
        N.check(self._lib.sdfo_grid_export_candidates(self.handle, _np_ptr(out["count"]),
                                                      _np_ptr(out["phi"]), _np_ptr(out["normal"]),
                                                      _np_ptr(out["branch"])))
        return out

    def attach_candidates(self, stride, count, phi, normal, branch) -> None:
        """Contact-aware candidates for a grid made from host data (e.g. a
        contact-aware SDFO file); stored-voxel order as export_candidates."""
        n = self.stored_voxels
        cnt = np.ascontiguousarray(count, np.uint8).reshape(n)
        ph = np.ascontiguousarray(phi, np.float64).reshape(n * stride)
        nr = np.ascontiguousarray(normal, np.float64).reshape(n * stride * 3)
        br = np.ascontiguousarray(branch, np.int32).reshape(n * stride)
        N.check(self._lib.sdfo_grid_attach_candidates(self.handle, int(stride), _np_ptr(cnt),
                                                      _np_ptr(ph), _np_ptr(nr), _np_ptr(br)))
        self._refresh_info()

    def query_candidates(self, points, mode=None, stream=None) -> dict:
        """queryFast with its candidate list (SdfFastQueryResult): dict of CUDA
        tensors gap (N,), normal (N,3), witness (N,3), valid (N,), ncand (N,),
        kgap (N,8), knormal (N,8,3), kwitness (N,8,3), kbranch (N,8)."""
        torch = _torch()
        pts = points.contiguous().reshape(-1, 3)
        if pts.dtype != torch.float32 or not pts.is_cuda:
            raise ValueError("points must be a CUDA float32 tensor")
        n = pts.shape[0]
        d = pts.device
        f = dict(dtype=torch.float32, device=d)
        out = dict(gap=torch.empty(n, **f), normal=torch.empty((n, 3), **f),
                   witness=torch.empty((n, 3), **f),
                   valid=torch.empty(n, dtype=torch.uint8, device=d),
                   ncand=torch.empty(n, dtype=torch.int32, device=d), kgap=torch.empty((n, 8), **f),
                   knormal=torch.empty((n, 8, 3), **f), kwitness=torch.empty((n, 8, 3), **f),
                   kbranch=torch.empty((n, 8), dtype=torch.int32, device=d))
        m = self.mode if mode is None else N.mode_id(mode)
        N.check(self._lib.sdfo_query_candidates(
            self.handle, m, _t_ptr(pts), n, _t_ptr(out["gap"]), _t_ptr(out["normal"]),
            _t_ptr(out["witness"]), _t_ptr(out["valid"]), _t_ptr(out["ncand"]), _t_ptr(out["kgap"]),
            _t_ptr(out["knormal"]), _t_ptr(out["kwitness"]), _t_ptr(out["kbranch"]),
            _stream_ptr(stream)))
        return out

    @classmethod
    def build_sparse_batched(cls, meshes, mode=N.TRILINEAR, stream=None) -> list:
        """Many SdfBuilder::buildSparse calls in one batched build
        (sdfo_grid_build_sparse_batched): ``meshes`` is a list of dicts with
        ``verts``, ``tris`` and the build_sparse keyword arguments (same
        block_dim for all).  Returns one SdfGrid per mesh; the grids share one
        device allocation."""
        lib = N.load()
        keep = []
        descs = (N.MeshDesc * len(meshes))()
        for i, m in enumerate(meshes):
            v, t = cls._mesh(m["verts"], m["tris"])
            keep.append((v, t))
            p = N.SparseBuildParams(
                N.BuildParams(m.get("padding", 0.1), m.get("voxel_size", 0.0),
                              m.get("target_resolution", 128), m.get("max_resolution", 512)),
                m.get("block_dim", 8), m.get("halo_voxels", 2), m.get("band_voxels", 8),
                1 if m.get("store_hessian", True) else 0, m.get("band_distance", 0.0))
            descs[i] = N.MeshDesc(_np_ptr(v), len(v), _np_ptr(t), len(t), p)
        out = (ctypes.c_void_p * len(meshes))()
        N.check(lib.sdfo_grid_build_sparse_batched(descs, len(meshes), _stream_ptr(stream), out))
        return [cls(out[i], mode) for i in range(len(meshes))]

    def build_stats(self) -> dict:
        s = N.BuildStats()
        N.check(self._lib.sdfo_grid_build_stats(self.handle, ctypes.byref(s)))
        return {k: getattr(s, k) for k, _ in N.BuildStats._fields_}

    # ----------------------------------------------------- host data in/out
    @staticmethod
    def _info_from_spec(spec: dict, layout: int) -> N.GridInfo:
        info = N.GridInfo()
        for a in range(3):
            info.bmin[a] = float(spec["bmin"][a])
            info.bmax[a] = float(spec["bmax"][a]) if "bmax" in spec else float(
                spec["bmin"][a] + spec["shape"][a] * spec["voxel"][a])
            info.voxel[a] = float(spec["voxel"][a])
            info.shape[a] = int(spec["shape"][a])
        info.layout = layout
        return info

    @classmethod
    def from_dense(cls, spec: dict, phi, normal, hessian=None, witness=None,
                   mode=N.TRILINEAR) -> "SdfGrid":
        """SdfOracle(SdfData): FP64 arrays in x-fastest order."""
        info = cls._info_from_spec(spec, N.LAYOUT_DENSE)
        n = int(np.prod(spec["shape"]))
        phi = np.ascontiguousarray(phi, np.float64).reshape(n)
        normal = np.ascontiguousarray(normal, np.float64).reshape(n, 3)
        hessian = None if hessian is None else np.ascontiguousarray(hessian, np.float64).reshape(n, 6)
        witness = None if witness is None else np.ascontiguousarray(witness, np.float64).reshape(n, 3)
        out = ctypes.c_void_p()
        lib = N.load()
        N.check(lib.sdfo_grid_create_dense(ctypes.byref(info), _np_ptr(phi), _np_ptr(normal),
                                           _np_ptr(hessian), _np_ptr(witness), _stream_ptr(),
                                           ctypes.byref(out)))
        return cls(out.value, mode)

    @classmethod
    def from_sparse(cls, spec: dict, block_dim: int, ijk, phi, normal, hessian=None,
                    halo_voxels=2, band_distance=0.0, mode=N.TRILINEAR) -> "SdfGrid":
        """SdfOracle(SparseSdfData): blocks (B,3), phi (B,V), normal (B,V,3) FP32."""
        info = cls._info_from_spec(spec, N.LAYOUT_SPARSE)
        info.block_dim = int(block_dim)
        info.halo_voxels = int(halo_voxels)
        info.band_distance = float(band_distance)
        ijk = np.ascontiguousarray(ijk, np.int32).reshape(-1, 3)
        info.block_count = len(ijk)
        V = block_dim ** 3
        phi = np.ascontiguousarray(phi, np.float32).reshape(len(ijk), V)
        normal = np.ascontiguousarray(normal, np.float32).reshape(len(ijk), V, 3)
        hessian = None if hessian is None else np.ascontiguousarray(hessian, np.float32).reshape(
            len(ijk), V, 6)
        out = ctypes.c_void_p()
        lib = N.load()
        N.check(lib.sdfo_grid_create_sparse(ctypes.byref(info), _np_ptr(ijk), _np_ptr(phi),
                                            _np_ptr(normal), _np_ptr(hessian), _stream_ptr(),
                                            ctypes.byref(out)))
        return cls(out.value, mode)

    def to_fp16(self) -> "SdfGrid":
        out = ctypes.c_void_p()
        N.check(self._lib.sdfo_grid_to_fp16(self.handle, _stream_ptr(), ctypes.byref(out)))
        return SdfGrid(out.value, self.mode)

    def export_dense(self) -> dict:
        n = self.stored_voxels
        phi = np.zeros(n)
        nrm = np.zeros((n, 3))
        hes = np.zeros((n, 6))
        wit = np.zeros((n, 3))
        _torch().cuda.synchronize()
        N.check(self._lib.sdfo_grid_export_dense(self.handle, _np_ptr(phi), _np_ptr(nrm),
                                                 _np_ptr(hes), _np_ptr(wit)))
        return dict(phi=phi, normal=nrm, hessian=hes, witness=wit)

    def export_sparse(self) -> dict:
        B, V = self.block_count, self.block_dim ** 3
        ijk = np.zeros((B, 3), np.int32)
        phi = np.zeros((B, V), np.float32)
        nrm = np.zeros((B, V, 3), np.float32)
        hes = np.zeros((B, V, 6), np.float32)
        _torch().cuda.synchronize()
        N.check(self._lib.sdfo_grid_export_sparse(self.handle, _np_ptr(ijk), _np_ptr(phi),
                                                  _np_ptr(nrm), _np_ptr(hes)))
        return dict(ijk=ijk, phi=phi, normal=nrm, hessian=hes if self.has_hessian else None)

    def payload(self):
        """A torch copy (stored_voxels, 4) float32 of the query payload {phi, n}."""
        torch = _torch()
        t = torch.empty((self.stored_voxels, 4), dtype=torch.float32, device="cuda")
        N.check(self._lib.sdfo_grid_copy_payload(self.handle, _t_ptr(t), _stream_ptr()))
        return t

    def view(self, payload) -> "SdfGrid":
        """A grid sharing this grid's structure but reading ``payload`` (a CUDA
        float32 (stored_voxels, 4) tensor); the view keeps the tensor alive."""
        torch = _torch()
        if payload.dtype != torch.float32 or not payload.is_cuda or not payload.is_contiguous():
            raise ValueError("payload must be a contiguous CUDA float32 tensor")
        if tuple(payload.shape) != (self.stored_voxels, 4):
            raise ValueError(f"payload must have shape ({self.stored_voxels}, 4)")
        out = ctypes.c_void_p()
        N.check(self._lib.sdfo_grid_create_view(self.handle, _t_ptr(payload), ctypes.byref(out)))
        return SdfGrid(out.value, self.mode, _keepalive=(self, payload))

    # -------------------------------------------------------------- queries
    def query_tensors(self, points, mode=None, unit=False, witness=False, valid=True,
                      hess=False, stream=None) -> dict:
        """Device path: points (N,3) CUDA float32/float64 tensor -> dict of CUDA
        tensors gap (N,), grad (N,3) [, unit (N,3), witness (N,3), valid (N,)
        uint8, hess (N,3,3)]."""
        torch = _torch()
        if not points.is_cuda:
            raise ValueError("points must be a CUDA tensor")
        if points.dtype not in (torch.float32, torch.float64):
            raise ValueError("points must be float32 or float64")
        pts = points.contiguous().reshape(-1, 3)
        n = pts.shape[0]
        dev = pts.device
        out = dict(gap=torch.empty(n, dtype=torch.float32, device=dev),
                   grad=torch.empty((n, 3), dtype=torch.float32, device=dev))
        if unit:
            out["unit"] = torch.empty((n, 3), dtype=torch.float32, device=dev)
        if witness:
            out["witness"] = torch.empty((n, 3), dtype=torch.float32, device=dev)
        if valid:
            out["valid"] = torch.empty(n, dtype=torch.uint8, device=dev)
        if hess:
            out["hess"] = torch.empty((n, 3, 3), dtype=torch.float32, device=dev)
        m = self.mode if mode is None else N.mode_id(mode)
        N.check(self._lib.sdfo_query(self.handle, m, _t_ptr(pts),
                                     1 if pts.dtype == torch.float64 else 0, n,
                                     _t_ptr(out["gap"]), _t_ptr(out["grad"]),
                                     _t_ptr(out.get("unit")), _t_ptr(out.get("witness")),
                                     _t_ptr(out.get("valid")), _t_ptr(out.get("hess")),
                                     _stream_ptr(stream)))
        return out

    def query_host(self, points: np.ndarray, mode=None) -> dict:
        """Host path through sdfo_query_host (copies in and out, synchronous)."""
        pts = np.ascontiguousarray(points)
        if pts.dtype not in (np.float32, np.float64):
            pts = pts.astype(np.float64)
        pts = pts.reshape(-1, 3)
        n = len(pts)
        gap = np.zeros(n, np.float32)
        grad = np.zeros((n, 3), np.float32)
        unit = np.zeros((n, 3), np.float32)
        wit = np.zeros((n, 3), np.float32)
        valid = np.zeros(n, np.uint8)
        m = self.mode if mode is None else N.mode_id(mode)
        N.check(self._lib.sdfo_query_host(self.handle, m, _np_ptr(pts),
                                          1 if pts.dtype == np.float64 else 0, n, _np_ptr(gap),
                                          _np_ptr(grad), _np_ptr(unit), _np_ptr(wit),
                                          _np_ptr(valid), _stream_ptr()))
        return dict(gap=gap, grad=grad, unit=unit, witness=wit, valid=valid.astype(bool))

    def query_batch(self, Y_local):
        """TrilinearSDFGrid.query_batch duck type (sdf_grid.py:138-204):
        (g, raw_grad, grad_norm, unit_normal, valid) as float64 / bool NumPy
        arrays; invalid points get g 0, grad 0, unit (0,0,1); a gradient with
        norm <= 1e-30 gets unit (0,0,1)."""
        Y = np.asarray(Y_local, dtype=np.float64).reshape(-1, 3)
        r = self.query_host(Y)
        valid = r["valid"]
        g = np.where(valid, r["gap"].astype(np.float64), 0.0)
        raw = np.where(valid[:, None], r["grad"].astype(np.float64), 0.0)
        gn = np.sqrt(np.einsum("ij,ij->i", raw, raw))
        unit = np.zeros((len(Y), 3))
        unit[:, 2] = 1.0
        ok = valid & (gn > 1e-30)
        unit[ok] = raw[ok] / gn[ok, None]
        return g, raw, gn, unit, valid

    def query(self, y_local):
        """TrilinearSDFGrid.query duck type for one point."""
        g, raw, gn, unit, valid = self.query_batch(np.asarray(y_local, np.float64).reshape(1, 3))
        if not valid[0]:
            return 0.0, np.zeros(3), 0.0, np.array([0.0, 0.0, 1.0]), False
        return float(g[0]), raw[0], float(gn[0]), unit[0], True

    def query_backward(self, points, dgap=None, dgrad=None, mode=None, dgrid=None,
                       want_points=True, stream=None):
        """Backward of the Trilinear/Tricubic query: returns dL/dpoints (N,3) and
        accumulates dL/dpayload into ``dgrid`` ((stored_voxels, 4) float32)."""
        torch = _torch()
        pts = points.contiguous().reshape(-1, 3)
        if pts.dtype != torch.float32:
            raise ValueError("backward takes float32 points")
        n = pts.shape[0]
        dpts = torch.empty((n, 3), dtype=torch.float32, device=pts.device) if want_points else None
        m = self.mode if mode is None else N.mode_id(mode)
        N.check(self._lib.sdfo_query_backward(
            self.handle, m, _t_ptr(pts), n,
            _t_ptr(None if dgap is None else dgap.contiguous()),
            _t_ptr(None if dgrad is None else dgrad.contiguous()),
            _t_ptr(dpts), _t_ptr(dgrid), _stream_ptr(stream)))
        return dpts

    def query_linearize(self, points, mode=None, stream=None):
        """Forward that also keeps the local linearisation for reverse mode:
        dict gap (N,), grad (N,3), valid (N,) uint8 and hess6 (N,6) = the
        interpolant's symmetric Hessian {xx, xy, xz, yy, yz, zz}."""
        torch = _torch()
        pts = points.contiguous().reshape(-1, 3)
        if pts.dtype != torch.float32:
            raise ValueError("query_linearize takes float32 points")
        n = pts.shape[0]
        dev = pts.device
        out = dict(gap=torch.empty(n, dtype=torch.float32, device=dev),
                   grad=torch.empty((n, 3), dtype=torch.float32, device=dev),
                   valid=torch.empty(n, dtype=torch.uint8, device=dev),
                   hess6=torch.empty((n, 6), dtype=torch.float32, device=dev))
        m = self.mode if mode is None else N.mode_id(mode)
        N.check(self._lib.sdfo_query_linearize(
            self.handle, m, _t_ptr(pts), n, _t_ptr(out["gap"]), _t_ptr(out["grad"]),
            _t_ptr(out["valid"]), _t_ptr(out["hess6"]), _stream_ptr(stream)))
        return out

    def query_backward_saved(self, points, saved, dgap=None, dgrad=None, mode=None, dgrid=None,
                             want_points=True, stream=None):
        """Backward from ``saved`` = query_linearize(points) (or a dict with at
        least ``valid`` when only ``dgrid`` is wanted): returns dL/dpoints
        (N,3) or None, and accumulates dL/dpayload into ``dgrid``."""
        torch = _torch()
        pts = points.contiguous().reshape(-1, 3)
        if pts.dtype != torch.float32:
            raise ValueError("backward takes float32 points")
        n = pts.shape[0]
        dpts = torch.empty((n, 3), dtype=torch.float32, device=pts.device) if want_points else None
        m = self.mode if mode is None else N.mode_id(mode)
        N.check(self._lib.sdfo_query_backward_saved(
            self.handle, m, _t_ptr(pts), n, _t_ptr(saved.get("grad")),
            _t_ptr(saved.get("hess6")), _t_ptr(saved.get("valid")),
            _t_ptr(None if dgap is None else dgap.contiguous()),
            _t_ptr(None if dgrad is None else dgrad.contiguous()),
            _t_ptr(dpts), _t_ptr(dgrid), _stream_ptr(stream)))
        return dpts

    # ----------------------------------------------------------------- io
    @classmethod
    def load(cls, path: str, mode=N.TRILINEAR, expect: str = "any", stream=None) -> "SdfGrid":
        """SdfOracle::loadFromFile (SdfOracle.cpp:165-172) straight onto the
        device; ``expect`` "dense" / "sparse" give loadSdf / loadSparseSdf
        (SdfIO.cpp:277-523) and their errors (SdfoError with the reference's
        message)."""
        kinds = {"any": N.FILE_ANY, "dense": N.FILE_DENSE, "sparse": N.FILE_SPARSE}
        if expect not in kinds:
            raise ValueError(f"expect must be one of {sorted(kinds)}")
        lib = N.load()
        out = ctypes.c_void_p()
        N.check(lib.sdfo_grid_load_file(os.fsencode(path), kinds[expect], _stream_ptr(stream),
                                        ctypes.byref(out)))
        return cls(out.value, mode)

    def save(self, path: str, stream=None) -> bool:
        """saveSdf / saveSparseSdf (SdfIO.cpp:93-275) of the device grid:
        False when the file cannot be opened or written, as the reference."""
        rc = self._lib.sdfo_grid_save_file(self.handle, os.fsencode(path), _stream_ptr(stream))
        if rc == N.SDFO_ERR_IO:
            return False
        N.check(rc)
        return True

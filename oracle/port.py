"""ctypes binding to the oracle restatement oracle/_port/libsdfo_port.so
(oracle/sdfo_port.c) plus its NumPy drivers.

TEST INFRASTRUCTURE ONLY: the checker the CUDA kernels are compared against.
Imported by tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg;
never by the product package.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_port", "libsdfo_port.so")

FIRST_ORDER, SECOND_ORDER, TRILINEAR, TRICUBIC = 0, 1, 2, 3

_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_int64
_D = ctypes.c_double


class _Spec(ctypes.Structure):
    _fields_ = [("bmin", _D * 3), ("bmax", _D * 3), ("voxel", _D * 3), ("shape", _I * 3)]


_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"oracle restatement not built: {LIB_PATH}")
        L = ctypes.CDLL(LIB_PATH)
        L.port_setup_grid.argtypes = [_P, _I, _D, _D, _I, _I, ctypes.POINTER(_Spec)]
        L.port_snap_resolution.argtypes = [_I, _I]
        L.port_snap_resolution.restype = _I
        L.port_bvh_build.argtypes = [_P, _I, _P, _I]
        L.port_bvh_build.restype = _P
        L.port_bvh_free.argtypes = [_P]
        L.port_signed_nearest.argtypes = [_P, _P, _L, _P, _P, _P, _P, _P]
        L.port_nearest_distance.argtypes = [_P, _P, _L, _P]
        L.port_traversal_counts.argtypes = [_P, _P, _L, _P]
        L.port_build_dense.argtypes = [_P, ctypes.POINTER(_Spec), _P, _P, _P, _P]
        L.port_dense_hessian.argtypes = [ctypes.POINTER(_Spec), _P, _P]
        L.port_sparse_activate.argtypes = [_P, ctypes.POINTER(_Spec), _I, _I, _D, _P]
        L.port_sparse_activate.restype = _I
        L.port_sparse_fill.argtypes = [_P, ctypes.POINTER(_Spec), _I, _I, _P, _P, _P]
        L.port_sparse_hessian.argtypes = [ctypes.POINTER(_Spec), _I, _I, _P, _P, _P]
        L.port_query_dense.argtypes = [ctypes.POINTER(_Spec), _P, _P, _P, _I, _P, _L, _P, _P,
                                       _P, _P, _P, _P]
        L.port_query_sparse.argtypes = [ctypes.POINTER(_Spec), _I, _I, _P, _P, _P, _P, _I, _P,
                                        _L, _P, _P, _P, _P, _P, _P]
        L.port_set_threads.argtypes = [_I]
        L.port_ca_prepare.restype = _P
        L.port_ca_prepare.argtypes = [_P, _I, _P, _I, _P, ctypes.POINTER(_Spec), _I, _I, _D]
        L.port_ca_free.argtypes = [_P]
        L.port_ca_dense.argtypes = [_P, _I, _D, _D, _P, _P, _P, _P, _P, _P, _P]
        L.port_ca_sparse_activate.restype = _I
        L.port_ca_sparse_activate.argtypes = [_P, _I, _D, _P]
        L.port_ca_sparse_fill.argtypes = [_P, _I, _I, _P, _I, _D, _D, _P, _P, _P, _P, _P, _P]
        L.port_ca_query_dense.argtypes = [ctypes.POINTER(_Spec), _I, _P, _P, _P, _P, _P, _L, _P,
                                          _P, _P, _P, _P, _P, _P, _P, _P]
        L.port_ca_query_sparse.argtypes = [ctypes.POINTER(_Spec), _I, _I, _P, _I, _P, _P, _P, _P,
                                           _P, _L, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def set_threads(n: int) -> None:
    lib().port_set_threads(int(n))


class GridSpec(dict):
    """bmin, bmax, voxel (float64 (3,)) and shape (nx, ny, nz)."""

    def to_c(self) -> _Spec:
        s = _Spec()
        for a in range(3):
            s.bmin[a] = float(self["bmin"][a])
            s.bmax[a] = float(self["bmax"][a])
            s.voxel[a] = float(self["voxel"][a])
            s.shape[a] = int(self["shape"][a])
        return s

    @staticmethod
    def from_c(s: _Spec) -> "GridSpec":
        return GridSpec(bmin=np.array(s.bmin[:]), bmax=np.array(s.bmax[:]),
                        voxel=np.array(s.voxel[:]), shape=tuple(int(x) for x in s.shape))


def snap_resolution(n: int, max_res: int) -> int:
    return int(lib().port_snap_resolution(int(n), int(max_res)))


def setup_grid(verts, padding=0.1, voxel_size=0.0, target_resolution=128,
               max_resolution=512) -> GridSpec:
    v = np.ascontiguousarray(verts, np.float64).reshape(-1, 3)
    s = _Spec()
    lib().port_setup_grid(_ptr(v), len(v), padding, voxel_size, target_resolution,
                          max_resolution, ctypes.byref(s))
    return GridSpec.from_c(s)


class Bvh:
    def __init__(self, verts, tris):
        self.v = np.ascontiguousarray(verts, np.float64).reshape(-1, 3)
        self.t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
        self.h = lib().port_bvh_build(_ptr(self.v), len(self.v), _ptr(self.t), len(self.t))

    def __del__(self):
        if getattr(self, "h", None) and _lib is not None:
            _lib.port_bvh_free(self.h)
            self.h = None

    def signed_nearest(self, pts):
        p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        n = len(p)
        sd = np.zeros(n)
        cp = np.zeros((n, 3))
        fn = np.zeros((n, 3))
        tri = np.zeros(n, np.int32)
        hits = np.zeros(n, np.int32)
        lib().port_signed_nearest(self.h, _ptr(p), n, _ptr(sd), _ptr(cp), _ptr(fn), _ptr(tri),
                                  _ptr(hits))
        return dict(sd=sd, cp=cp, fn=fn, tri=tri, hits=hits)

    def traversal_counts(self, pts):
        """[nodes entered past the nearest search's cut, closest-point tests,
        ray-box tests, ray-triangle tests] summed over the points."""
        p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        c = np.zeros(4, np.int64)
        lib().port_traversal_counts(self.h, _ptr(p), len(p), _ptr(c))
        return c

    def nearest_distance(self, pts):
        p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
        d = np.zeros(len(p))
        lib().port_nearest_distance(self.h, _ptr(p), len(p), _ptr(d))
        return d


def build_dense(verts, tris, padding=0.1, voxel_size=0.0, target_resolution=128,
                max_resolution=512):
    """SdfBuilder::build restated: returns spec and FP64 phi (N,), normal (N,3),
    hessian (N,6), witness (N,3) in x-fastest order."""
    spec = setup_grid(verts, padding, voxel_size, target_resolution, max_resolution)
    bvh = Bvh(verts, tris)
    n = int(np.prod(spec["shape"]))
    phi = np.zeros(n)
    nrm = np.zeros((n, 3))
    hes = np.zeros((n, 6))
    wit = np.zeros((n, 3))
    s = spec.to_c()
    lib().port_build_dense(bvh.h, ctypes.byref(s), _ptr(phi), _ptr(nrm), _ptr(hes), _ptr(wit))
    return dict(spec=spec, phi=phi, normal=nrm, hessian=hes, witness=wit)


def resolve_band(spec: GridSpec, band_voxels: int, band_distance: float) -> float:
    h = float(np.max(spec["voxel"]))
    return band_distance if band_distance > 0.0 else float(band_voxels) * h


def build_sparse(verts, tris, padding=0.1, voxel_size=0.0, target_resolution=128,
                 max_resolution=512, block_dim=8, halo_voxels=2, band_voxels=8,
                 band_distance=0.0, store_hessian=True):
    """SdfBuilder::buildSparse restated: blocks in (bk, bj, bi) order with FP32
    phi (B,V), normal (B,V,3) and hessian (B,V,6)."""
    spec = setup_grid(verts, padding, voxel_size, target_resolution, max_resolution)
    bvh = Bvh(verts, tris)
    band = resolve_band(spec, band_voxels, band_distance)
    nb = [(spec["shape"][a] + block_dim - 1) // block_dim for a in range(3)]
    active = np.zeros(nb[0] * nb[1] * nb[2], np.uint8)
    s = spec.to_c()
    lib().port_sparse_activate(bvh.h, ctypes.byref(s), block_dim, halo_voxels, band,
                               _ptr(active))
    lin = np.nonzero(active)[0]
    ijk = np.stack([lin % nb[0], (lin // nb[0]) % nb[1], lin // (nb[0] * nb[1])], -1)
    ijk = np.ascontiguousarray(ijk, np.int32)
    V = block_dim ** 3
    B = len(ijk)
    phi = np.zeros((B, V), np.float32)
    nrm = np.zeros((B, V, 3), np.float32)
    lib().port_sparse_fill(bvh.h, ctypes.byref(s), block_dim, B, _ptr(ijk), _ptr(phi), _ptr(nrm))
    hes = np.zeros((B, V, 6), np.float32)
    if store_hessian:
        lib().port_sparse_hessian(ctypes.byref(s), block_dim, B, _ptr(ijk), _ptr(nrm), _ptr(hes))
    return dict(spec=spec, block_dim=block_dim, halo=halo_voxels, band=band, ijk=ijk, phi=phi,
                normal=nrm, hessian=hes if store_hessian else None, active=active)


def sparse_hessian(spec: GridSpec, block_dim, ijk, normal):
    ijk = np.ascontiguousarray(ijk, np.int32)
    nrm = np.ascontiguousarray(normal, np.float32)
    hes = np.zeros(nrm.shape[:-1] + (6,), np.float32)
    s = spec.to_c()
    lib().port_sparse_hessian(ctypes.byref(s), block_dim, len(ijk), _ptr(ijk), _ptr(nrm),
                              _ptr(hes))
    return hes


def dense_hessian(spec: GridSpec, normal):
    nrm = np.ascontiguousarray(normal, np.float64)
    hes = np.zeros((len(nrm), 6))
    s = spec.to_c()
    lib().port_dense_hessian(ctypes.byref(s), _ptr(nrm), _ptr(hes))
    return hes


def _query_out(n):
    return (np.zeros(n), np.zeros((n, 3)), np.zeros((n, 3)), np.zeros((n, 3)),
            np.zeros(n, np.uint8), np.zeros((n, 3, 3)))


def query_dense(spec: GridSpec, phi, normal, hessian, mode: int, pts):
    """FP64 queries on a dense grid: dict(gap, grad, unit, witness, valid, hess)."""
    p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
    n = len(p)
    phi = np.ascontiguousarray(phi, np.float64)
    nrm = np.ascontiguousarray(normal, np.float64)
    hes = None if hessian is None else np.ascontiguousarray(hessian, np.float64)
    gap, grad, unit, wit, valid, hs = _query_out(n)
    s = spec.to_c()
    lib().port_query_dense(ctypes.byref(s), _ptr(phi), _ptr(nrm), _ptr(hes), int(mode), _ptr(p),
                           n, _ptr(gap), _ptr(grad), _ptr(unit), _ptr(wit), _ptr(valid),
                           _ptr(hs))
    return dict(gap=gap, grad=grad, unit=unit, witness=wit, valid=valid.astype(bool), hess=hs)


def query_sparse(spec: GridSpec, block_dim, ijk, phi, normal, hessian, mode: int, pts):
    p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
    n = len(p)
    ijk = np.ascontiguousarray(ijk, np.int32)
    phi = np.ascontiguousarray(phi, np.float32)
    nrm = np.ascontiguousarray(normal, np.float32)
    hes = None if hessian is None else np.ascontiguousarray(hessian, np.float32)
    gap, grad, unit, wit, valid, hs = _query_out(n)
    s = spec.to_c()
    lib().port_query_sparse(ctypes.byref(s), block_dim, len(ijk), _ptr(ijk), _ptr(phi),
                            _ptr(nrm), _ptr(hes), int(mode), _ptr(p), n, _ptr(gap), _ptr(grad),
                            _ptr(unit), _ptr(wit), _ptr(valid), _ptr(hs))
    return dict(gap=gap, grad=grad, unit=unit, witness=wit, valid=valid.astype(bool), hess=hs)


# ---------------------------------------------------------------------------
# contact-aware builds and queries (SdfBuilder.cpp:27-359, 416-821;
# SdfOracle.cpp:269-431)
# ---------------------------------------------------------------------------
def build_contact_aware(verts, tris, corner_normals, padding=0.1, voxel_size=0.0,
                        target_resolution=128, max_resolution=512, max_candidates=4,
                        feature_distance_tolerance=0.0, normal_merge_angle_degrees=5.0,
                        tile_dim=8, use_tile_acceleration=True, store_hessian=True, sparse=False,
                        block_dim=8, halo_voxels=2, band_voxels=8, band_distance=0.0):
    """SdfBuilder::buildContactAware / buildSparseContactAware restated.
    Dense: phi, normal, witness (primary candidate), hessian, count (N,),
    cphi (N,s), cnormal (N,s,3), cbranch (N,s).  Sparse: ijk, phi (B,V),
    normal (B,V,3), hessian (B,V,6), count (B,V), cphi (B,V,s), cnormal
    (B,V,s,3), cbranch (B,V,s) -- FP32."""
    v = np.ascontiguousarray(verts, np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(tris, np.int32).reshape(-1, 3)
    cn = np.ascontiguousarray(corner_normals, np.float64).reshape(-1, 3, 3)
    spec = setup_grid(v, padding, voxel_size, target_resolution, max_resolution)
    h = float(np.max(spec["voxel"]))
    tol = feature_distance_tolerance if feature_distance_tolerance > 0.0 else 1.5 * h
    cos_merge = float(np.cos(normal_merge_angle_degrees * np.arccos(-1.0) / 180.0))
    stride = max(0, min(max_candidates, 8))
    s = spec.to_c()
    if not sparse:
        influence = tol + 2.0 * h
    else:
        band = band_distance if band_distance > 0.0 else float(band_voxels) * h
        activation = band + float(halo_voxels) * h
        influence = max(activation, tol + 2.0 * h)
    ctx = lib().port_ca_prepare(_ptr(v), len(v), _ptr(t), len(t), _ptr(cn), ctypes.byref(s),
                                tile_dim, 1 if use_tile_acceleration else 0, influence)
    try:
        if not sparse:
            n = int(np.prod(spec["shape"]))
            out = dict(spec=spec, stride=stride, count=np.zeros(n, np.uint8),
                       cphi=np.zeros((n, stride)), cnormal=np.zeros((n, stride, 3)),
                       cbranch=np.zeros((n, stride), np.int32), phi=np.zeros(n),
                       normal=np.zeros((n, 3)), witness=np.zeros((n, 3)))
            lib().port_ca_dense(ctx, stride, tol, cos_merge, _ptr(out["count"]), _ptr(out["cphi"]),
                                _ptr(out["cnormal"]), _ptr(out["cbranch"]), _ptr(out["phi"]),
                                _ptr(out["normal"]), _ptr(out["witness"]))
            out["hessian"] = dense_hessian(spec, out["normal"]) if store_hessian else None
            return out
        nb = [(spec["shape"][a] + block_dim - 1) // block_dim for a in range(3)]
        active = np.zeros(nb[0] * nb[1] * nb[2], np.uint8)
        lib().port_ca_sparse_activate(ctx, block_dim, activation, _ptr(active))
        lin = np.nonzero(active)[0]
        ijk = np.ascontiguousarray(
            np.stack([lin % nb[0], (lin // nb[0]) % nb[1], lin // (nb[0] * nb[1])], -1), np.int32)
        B, V = len(ijk), block_dim ** 3
        out = dict(spec=spec, stride=stride, block_dim=block_dim, halo=halo_voxels, band=band,
                   ijk=ijk, phi=np.zeros((B, V), np.float32), normal=np.zeros((B, V, 3), np.float32),
                   count=np.zeros((B, V), np.uint8), cphi=np.zeros((B, V, stride), np.float32),
                   cnormal=np.zeros((B, V, stride, 3), np.float32),
                   cbranch=np.zeros((B, V, stride), np.int32))
        lib().port_ca_sparse_fill(ctx, block_dim, B, _ptr(ijk), stride, tol, cos_merge,
                                  _ptr(out["phi"]), _ptr(out["normal"]), _ptr(out["count"]),
                                  _ptr(out["cphi"]), _ptr(out["cnormal"]), _ptr(out["cbranch"]))
        out["hessian"] = (sparse_hessian(spec, block_dim, ijk, out["normal"])
                          if store_hessian else None)
        return out
    finally:
        lib().port_ca_free(ctx)


def query_contact_aware(g: dict, pts):
    """queryFast(ContactAware) on a build_contact_aware result: gap, normal
    (gapNormal), witness, valid, ncand, and the candidates kgap (n,8),
    knormal (n,8,3), kwitness (n,8,3), kbranch (n,8).  Voxels without
    candidates take the FirstOrder query (SdfOracle.cpp:329, 385), as in the
    reference, with a single candidate of branch 0."""
    p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
    n = len(p)
    out = dict(gap=np.zeros(n), normal=np.zeros((n, 3)), witness=np.zeros((n, 3)),
               valid=np.zeros(n, np.uint8), ncand=np.zeros(n, np.int32),
               kgap=np.zeros((n, 8)), knormal=np.zeros((n, 8, 3)), kwitness=np.zeros((n, 8, 3)),
               kbranch=np.full((n, 8), -1, np.int32))
    s = g["spec"].to_c()
    cnt = np.ascontiguousarray(g["count"], np.uint8)
    br = np.ascontiguousarray(g["cbranch"], np.int32)
    if "ijk" in g:
        ijk = np.ascontiguousarray(g["ijk"], np.int32)
        lib().port_ca_query_sparse(ctypes.byref(s), g["block_dim"], len(ijk), _ptr(ijk), g["stride"],
                                   _ptr(cnt), _ptr(np.ascontiguousarray(g["cphi"], np.float32)),
                                   _ptr(np.ascontiguousarray(g["cnormal"], np.float32)), _ptr(br),
                                   _ptr(p), n, _ptr(out["valid"]), _ptr(out["gap"]),
                                   _ptr(out["normal"]), _ptr(out["witness"]), _ptr(out["ncand"]),
                                   _ptr(out["kgap"]), _ptr(out["knormal"]), _ptr(out["kwitness"]),
                                   _ptr(out["kbranch"]))
        first = query_sparse(g["spec"], g["block_dim"], ijk, g["phi"], g["normal"], None,
                             FIRST_ORDER, p)
    else:
        lib().port_ca_query_dense(ctypes.byref(s), g["stride"], _ptr(cnt),
                                  _ptr(np.ascontiguousarray(g["cphi"], np.float64)),
                                  _ptr(np.ascontiguousarray(g["cnormal"], np.float64)), _ptr(br),
                                  _ptr(p), n, _ptr(out["valid"]), _ptr(out["gap"]),
                                  _ptr(out["normal"]), _ptr(out["witness"]), _ptr(out["ncand"]),
                                  _ptr(out["kgap"]), _ptr(out["knormal"]), _ptr(out["kwitness"]),
                                  _ptr(out["kbranch"]))
        first = query_dense(g["spec"], g["phi"], g["normal"], None, FIRST_ORDER, p)
    out["valid"] = out["valid"].astype(bool)
    fo = out["valid"] & (out["ncand"] == 0)
    out["gap"][fo] = first["gap"][fo]
    out["normal"][fo] = first["unit"][fo]
    out["witness"][fo] = first["witness"][fo]
    out["ncand"][fo] = 1
    out["kgap"][fo, 0] = first["gap"][fo]
    out["knormal"][fo, 0] = first["unit"][fo]
    out["kwitness"][fo, 0] = first["witness"][fo]
    out["kbranch"][fo, 0] = 0
    return out

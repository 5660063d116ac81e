"""ctypes binding to oracle/_ref/libsdfo_ref.so -- the reference SdfOracle C++
sources compiled unmodified (see oracle/Makefile and oracle/ref_capi.cpp).

Test infrastructure only: used by tests/, the golden-fixture generator and the
CPU baseline of bench.py.  Never imported by the product package.
"""
from __future__ import annotations

import ctypes
import os
from dataclasses import dataclass

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_ref", "libsdfo_ref.so")

_P = ctypes.c_void_p
_I = ctypes.c_int
_L = ctypes.c_int64
_D = ctypes.c_double

_lib = None


def available() -> bool:
    return os.path.exists(LIB_PATH)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"reference oracle not built: {LIB_PATH}")
        L = ctypes.CDLL(LIB_PATH)
        L.ref_last_error.restype = ctypes.c_char_p
        L.ref_set_threads.argtypes = [_I]
        L.ref_max_threads.restype = _I
        L.ref_build_dense.restype = _P
        L.ref_build_dense.argtypes = [_P, _I, _P, _I, _D, _D, _I, _I, _P]
        L.ref_build_sparse.restype = _P
        L.ref_build_sparse.argtypes = [_P, _I, _P, _I, _D, _D, _I, _I, _I, _I, _I, _D, _I, _P]
        L.ref_load.restype = _P
        L.ref_load.argtypes = [ctypes.c_char_p]
        L.ref_save.restype = _I
        L.ref_save.argtypes = [_P, ctypes.c_char_p]
        L.ref_load_kind.restype = _P
        L.ref_load_kind.argtypes = [ctypes.c_char_p, _I, _P]
        L.ref_save_timed.restype = _I
        L.ref_save_timed.argtypes = [_P, ctypes.c_char_p, _P]
        L.ref_free.argtypes = [_P]
        L.ref_grid_info.argtypes = [_P, _P, _P, _P, _P, _P, _P, _P]
        L.ref_dense_export.argtypes = [_P, _P, _P, _P, _P]
        L.ref_sparse_export.argtypes = [_P, _P, _P, _P, _P]
        L.ref_query.argtypes = [_P, _I, _P, _L, _P, _P, _P, _P]
        L.ref_query_bench.restype = _D
        L.ref_query_bench.argtypes = [_P, _I, _P, _L, _P, _P]
        L.ref_signed_nearest.restype = _I
        L.ref_signed_nearest.argtypes = [_P, _I, _P, _I, _P, _L, _P, _P, _P, _P]
        L.ref_load_obj.restype = _I
        L.ref_load_obj.argtypes = [ctypes.c_char_p, _P, _P, _P, _P]
        L.ref_build_contact_aware.restype = _P
        L.ref_build_contact_aware.argtypes = [_P, _I, _P, _I, _P, _D, _D, _I, _I, _I, _D, _D, _I,
                                              _I, _I, _I, _I, _I, _I, _D, _P]
        L.ref_ca_stride.restype = _I
        L.ref_ca_stride.argtypes = [_P]
        L.ref_ca_export_dense.restype = _I
        L.ref_ca_export_dense.argtypes = [_P, _P, _P, _P, _P]
        L.ref_ca_export_sparse.restype = _I
        L.ref_ca_export_sparse.argtypes = [_P, _P, _P, _P, _P]
        L.ref_query_candidates.restype = _I
        L.ref_query_candidates.argtypes = [_P, _I, _P, _L, _P, _P, _P, _P, _P, _P, _P, _P, _P]
        L.ref_load_ca_surface.restype = _I
        L.ref_load_ca_surface.argtypes = [ctypes.c_char_p, _P, _P, _P, _P, _P]
        _lib = L
    return _lib


def _ptr(a):
    return None if a is None else a.ctypes.data


def set_threads(n: int) -> None:
    lib().ref_set_threads(int(n))


def max_threads() -> int:
    return int(lib().ref_max_threads())


@dataclass
class RefGrid:
    """Handle to a reference SdfOracle (dense or sparse)."""

    handle: int
    build_seconds: float = 0.0

    def __del__(self):
        if self.handle and _lib is not None:
            _lib.ref_free(self.handle)
            self.handle = 0

    def info(self):
        shape = np.zeros(3, np.int32)
        bmin = np.zeros(3)
        bmax = np.zeros(3)
        voxel = np.zeros(3)
        sp = np.zeros(1, np.int32)
        info = np.zeros(4, np.int32)
        band = np.zeros(1)
        lib().ref_grid_info(self.handle, _ptr(shape), _ptr(bmin), _ptr(bmax), _ptr(voxel),
                            _ptr(sp), _ptr(info), _ptr(band))
        return dict(shape=tuple(int(s) for s in shape), bmin=bmin, bmax=bmax, voxel=voxel,
                    sparse=bool(sp[0]), blocks=int(info[0]), block_dim=int(info[1]),
                    halo=int(info[2]), has_hessian=bool(info[3]), band=float(band[0]))

    def dense_arrays(self):
        inf = self.info()
        n = int(np.prod(inf["shape"]))
        phi = np.zeros(n)
        nrm = np.zeros((n, 3))
        hes = np.zeros((n, 6))
        wit = np.zeros((n, 3))
        rc = lib().ref_dense_export(self.handle, _ptr(phi), _ptr(nrm), _ptr(hes), _ptr(wit))
        if rc != 0:
            raise ValueError("not a dense grid")
        return dict(phi=phi, normal=nrm, hessian=hes, witness=wit)

    def sparse_arrays(self):
        inf = self.info()
        b, d = inf["blocks"], inf["block_dim"]
        v = d * d * d
        ijk = np.zeros((b, 3), np.int32)
        phi = np.zeros((b, v), np.float32)
        nrm = np.zeros((b, v, 3), np.float32)
        hes = np.zeros((b, v, 6), np.float32)
        rc = lib().ref_sparse_export(self.handle, _ptr(ijk), _ptr(phi), _ptr(nrm), _ptr(hes))
        if rc != 0:
            raise ValueError("not a sparse grid")
        return dict(ijk=ijk, phi=phi, normal=nrm, hessian=hes)

    def query(self, mode: int, pts: np.ndarray):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        n = len(pts)
        gap = np.zeros(n)
        nrm = np.zeros((n, 3))
        wit = np.zeros((n, 3))
        valid = np.zeros(n, np.uint8)
        lib().ref_query(self.handle, int(mode), _ptr(pts), n, _ptr(gap), _ptr(nrm), _ptr(wit),
                        _ptr(valid))
        return gap, nrm, wit, valid.astype(bool)

    def query_bench(self, mode: int, pts: np.ndarray):
        pts = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
        valid = np.zeros(1, np.int64)
        avg = np.zeros(1)
        sec = lib().ref_query_bench(self.handle, int(mode), _ptr(pts), len(pts), _ptr(valid),
                                    _ptr(avg))
        return float(sec), int(valid[0]), float(avg[0])

    def save(self, path: str) -> bool:
        return lib().ref_save(self.handle, path.encode()) == 0


def _err():
    return lib().ref_last_error().decode()


def _mesh(verts, tris):
    v = np.ascontiguousarray(verts, dtype=np.float64).reshape(-1, 3)
    t = np.ascontiguousarray(tris, dtype=np.int32).reshape(-1, 3)
    return v, t


def build_dense(verts, tris, padding=0.1, voxel_size=0.0, target_resolution=128,
                max_resolution=512) -> RefGrid:
    v, t = _mesh(verts, tris)
    sec = np.zeros(1)
    h = lib().ref_build_dense(_ptr(v), len(v), _ptr(t), len(t), padding, voxel_size,
                              target_resolution, max_resolution, _ptr(sec))
    if not h:
        raise RuntimeError(_err())
    return RefGrid(h, float(sec[0]))


def build_sparse(verts, tris, padding=0.1, voxel_size=0.0, target_resolution=128,
                 max_resolution=512, block_dim=8, halo_voxels=2, band_voxels=8,
                 band_distance=0.0, store_hessian=True) -> RefGrid:
    v, t = _mesh(verts, tris)
    sec = np.zeros(1)
    h = lib().ref_build_sparse(_ptr(v), len(v), _ptr(t), len(t), padding, voxel_size,
                               target_resolution, max_resolution, block_dim, halo_voxels,
                               band_voxels, band_distance, 1 if store_hessian else 0, _ptr(sec))
    if not h:
        raise RuntimeError(_err())
    return RefGrid(h, float(sec[0]))


def load(path: str) -> RefGrid:
    h = lib().ref_load(path.encode())
    if not h:
        raise RuntimeError(_err())
    return RefGrid(h)


def load_kind(path: str, kind: str = "any") -> RefGrid:
    """SdfOracle::loadFromFile ("any"), loadSdf ("dense") or loadSparseSdf
    ("sparse") (SdfIO.cpp:277-523); RuntimeError with the reference's message
    on failure; ``build_seconds`` holds the load's wall time."""
    sec = np.zeros(1)
    h = lib().ref_load_kind(path.encode(), {"any": 0, "dense": 1, "sparse": 2}[kind], _ptr(sec))
    if not h:
        raise RuntimeError(_err())
    return RefGrid(h, float(sec[0]))


def save_timed(g: "RefGrid", path: str):
    """saveSdf / saveSparseSdf: (ok, seconds)."""
    sec = np.zeros(1)
    rc = lib().ref_save_timed(g.handle, path.encode(), _ptr(sec))
    return rc == 0, float(sec[0])


def signed_nearest(verts, tris, pts):
    v, t = _mesh(verts, tris)
    p = np.ascontiguousarray(pts, dtype=np.float64).reshape(-1, 3)
    n = len(p)
    sd = np.zeros(n)
    cp = np.zeros((n, 3))
    fn = np.zeros((n, 3))
    tri = np.zeros(n, np.int32)
    rc = lib().ref_signed_nearest(_ptr(v), len(v), _ptr(t), len(t), _ptr(p), n, _ptr(sd),
                                  _ptr(cp), _ptr(fn), _ptr(tri))
    if rc != 0:
        raise RuntimeError(_err())
    return sd, cp, fn, tri


def load_obj(path: str):
    nv = np.zeros(1, np.int32)
    nt = np.zeros(1, np.int32)
    if lib().ref_load_obj(path.encode(), None, _ptr(nv), None, _ptr(nt)) != 0:
        raise RuntimeError(_err())
    v = np.zeros((int(nv[0]), 3))
    t = np.zeros((int(nt[0]), 3), np.int32)
    lib().ref_load_obj(path.encode(), _ptr(v), _ptr(nv), _ptr(t), _ptr(nt))
    return v, t


def build_contact_aware(verts, tris, corner_normals, padding=0.1, voxel_size=0.0,
                        target_resolution=128, max_resolution=512, max_candidates=4,
                        feature_distance_tolerance=0.0, normal_merge_angle_degrees=5.0,
                        tile_dim=8, use_tile_acceleration=True, store_hessian=True, sparse=False,
                        block_dim=8, halo_voxels=2, band_voxels=8, band_distance=0.0) -> "RefGrid":
    """SdfBuilder::buildContactAware / buildSparseContactAware
    (SdfBuilder.cpp:416-821) with ContactAwareBuilderParams' defaults."""
    v, t = _mesh(verts, tris)
    cn = np.ascontiguousarray(corner_normals, np.float64).reshape(-1, 3, 3)
    sec = np.zeros(1)
    h = lib().ref_build_contact_aware(
        _ptr(v), len(v), _ptr(t), len(t), _ptr(cn), padding, voxel_size, target_resolution,
        max_resolution, max_candidates, feature_distance_tolerance, normal_merge_angle_degrees,
        tile_dim, 1 if use_tile_acceleration else 0, 1 if store_hessian else 0,
        1 if sparse else 0, block_dim, halo_voxels, band_voxels, band_distance, _ptr(sec))
    if not h:
        raise RuntimeError(_err())
    return RefGrid(h, float(sec[0]))


def ca_arrays(g: "RefGrid"):
    """Candidate arrays of a contact-aware grid: stride, count, phi, normal,
    branch (dense: (N, s[, 3]) FP64; sparse: (B, V, s[, 3]) FP32)."""
    s = lib().ref_ca_stride(g.handle)
    info = g.info()
    if info["sparse"]:
        B, V = info["blocks"], info["block_dim"] ** 3
        cnt = np.zeros((B, V), np.uint8)
        phi = np.zeros((B, V, s), np.float32)
        nrm = np.zeros((B, V, s, 3), np.float32)
        br = np.zeros((B, V, s), np.int32)
        lib().ref_ca_export_sparse(g.handle, _ptr(cnt), _ptr(phi), _ptr(nrm), _ptr(br))
    else:
        N = int(np.prod(info["shape"]))
        cnt = np.zeros(N, np.uint8)
        phi = np.zeros((N, s))
        nrm = np.zeros((N, s, 3))
        br = np.zeros((N, s), np.int32)
        lib().ref_ca_export_dense(g.handle, _ptr(cnt), _ptr(phi), _ptr(nrm), _ptr(br))
    return dict(stride=s, count=cnt, phi=phi, normal=nrm, branch=br)


def query_candidates(g: "RefGrid", mode: int, pts):
    """queryFast with the candidate list (SdfFastQueryResult, SdfCommon.h:29-37)."""
    p = np.ascontiguousarray(pts, np.float64).reshape(-1, 3)
    n = len(p)
    out = dict(gap=np.zeros(n), normal=np.zeros((n, 3)), witness=np.zeros((n, 3)),
               valid=np.zeros(n, np.uint8), ncand=np.zeros(n, np.int32),
               kgap=np.zeros((n, 8)), knormal=np.zeros((n, 8, 3)), kwitness=np.zeros((n, 8, 3)),
               kbranch=np.zeros((n, 8), np.int32))
    lib().ref_query_candidates(g.handle, int(mode), _ptr(p), n, _ptr(out["gap"]),
                               _ptr(out["normal"]), _ptr(out["witness"]), _ptr(out["valid"]),
                               _ptr(out["ncand"]), _ptr(out["kgap"]), _ptr(out["knormal"]),
                               _ptr(out["kwitness"]), _ptr(out["kbranch"]))
    out["valid"] = out["valid"].astype(bool)
    return out


def load_ca_surface(path: str):
    """loadContactAwareSurfaceFile: verts (nv,3), tris (nt,3), corner normals (nt,3,3)."""
    nv = np.zeros(1, np.int32)
    nt = np.zeros(1, np.int32)
    if lib().ref_load_ca_surface(path.encode(), None, _ptr(nv), None, _ptr(nt), None) != 0:
        raise RuntimeError(_err())
    v = np.zeros((int(nv[0]), 3))
    t = np.zeros((int(nt[0]), 3), np.int32)
    cn = np.zeros((int(nt[0]), 3, 3))
    lib().ref_load_ca_surface(path.encode(), _ptr(v), _ptr(nv), _ptr(t), _ptr(nt), _ptr(cn))
    return v, t, cn

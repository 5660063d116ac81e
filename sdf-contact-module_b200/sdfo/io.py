"""The "SDFO" v0.1.0 binary grid file (reference plugins/SdfOracle/src/SdfIO.cpp).

The byte layout is the reference's, unchanged, so files move freely between
the reference (C++ saveSdf / loadSdf, Python TrilinearSDFGrid) and this
package:

  header, 128 bytes, little-endian (SdfIO.cpp:62-80):
    0  "SDFO"            4  u32 version = 100 (0.1.0)
    8  u32 nx, ny, nz    20 f64 bmin[3]     44 f64 bmax[3]    68 f64 voxel[3]
    92 u32 flags (bit0 Hessian, bit1 sparse blocks, bit2 contact-aware)
    96 reserved[32]: +0 u32 layout (1 dense, 2 sparse, 3 dense CA, 4 sparse CA)
       dense CA: +4 u32 stride
       sparse:   +4 u32 blockDim, +8 u32 halo, +12 u32 blockCount,
                 +16 f64 bandDistance, +24 u32 CA stride
  dense payload (SdfIO.cpp:128-180): f64 phi[N], f64 n[N][3], f64 H[N][6]
    (xx,xy,xz,yy,yz,zz), f64 witness[N][3]; CA: u32 count[N], f64 phi[N*s],
    f64 n[N*s][3], i32 branch[N*s]
  sparse payload per block (SdfIO.cpp:226-272): i32 bi,bj,bk,u32 0;
    f32 phi[V], f32 n[V][3], [f32 H[V][6]]; CA: u8 count[V], f32 phi[V*s],
    f32 n[V*s][3], i32 branch[V*s]

Errors are RuntimeError with the reference's std::runtime_error messages.
"""
from __future__ import annotations

import struct

import numpy as np

VERSION = 100
VERSION_STRING = "0.1.0"
FLAG_HESSIAN = 1
FLAG_SPARSE = 2
FLAG_CONTACT_AWARE = 4
LAYOUT_DENSE, LAYOUT_SPARSE, LAYOUT_DENSE_CA, LAYOUT_SPARSE_CA = 1, 2, 3, 4
MAX_CANDIDATES = 8
HEADER = struct.Struct("<4sI3I3d3d3dI32s")
assert HEADER.size == 128


def _header(spec, flags, reserved: bytes) -> bytes:
    return HEADER.pack(b"SDFO", VERSION, *[int(x) for x in spec["shape"]],
                       *[float(x) for x in spec["bmin"]], *[float(x) for x in spec["bmax"]],
                       *[float(x) for x in spec["voxel"]], flags, reserved.ljust(32, b"\0"))


def read_header(path: str) -> dict:
    try:
        f = open(path, "rb")
    except OSError:
        raise RuntimeError("Cannot open SdfOracle data file: " + path) from None
    with f:
        raw = f.read(128)
    if len(raw) != 128:
        raise RuntimeError("Failed to read SdfOracle data header")
    magic, version, nx, ny, nz, *rest = HEADER.unpack(raw)
    bmin, bmax, voxel = rest[0:3], rest[3:6], rest[6:9]
    flags, reserved = rest[9], rest[10]
    return dict(magic=magic, version=version, shape=(nx, ny, nz), bmin=np.array(bmin),
                bmax=np.array(bmax), voxel=np.array(voxel), flags=flags, reserved=reserved)


def _check_magic_version(h: dict) -> None:
    if h["magic"] != b"SDFO":
        raise RuntimeError("Invalid SdfOracle data magic number")
    if h["version"] != VERSION:
        raise RuntimeError(f"Unsupported SdfOracle data version: {h['version']} "
                           f"(only {VERSION_STRING} is supported)")


def _u32(b: bytes, off: int) -> int:
    return struct.unpack_from("<I", b, off)[0]


def is_valid_sdf(path: str) -> bool:
    """isValidSdf (SdfIO.cpp:527-537)."""
    try:
        h = read_header(path)
    except RuntimeError:
        return False
    return h["magic"] == b"SDFO" and h["version"] == VERSION


def is_sparse_sdf(path: str) -> bool:
    """isSparseSdf (SdfIO.cpp:539-552)."""
    try:
        h = read_header(path)
    except RuntimeError:
        return False
    if h["magic"] != b"SDFO" or h["version"] != VERSION:
        return False
    layout = _u32(h["reserved"], 0)
    return bool(h["flags"] & FLAG_SPARSE) and layout in (LAYOUT_SPARSE, LAYOUT_SPARSE_CA)


class _Reader:
    def __init__(self, f, err: str):
        self.f = f
        self.err = err

    def arr(self, dtype, count):
        nbytes = np.dtype(dtype).itemsize * count
        b = self.f.read(nbytes)
        if len(b) != nbytes:
            raise RuntimeError(self.err)
        return np.frombuffer(b, dtype=dtype, count=count).copy()


def load_dense(path: str) -> dict:
    """loadSdf (SdfIO.cpp:279-394)."""
    h = read_header(path)
    _check_magic_version(h)
    if h["flags"] & FLAG_SPARSE:
        raise RuntimeError("SdfOracle data file uses sparse layout; call loadSparseSdf")
    layout = _u32(h["reserved"], 0)
    if layout not in (LAYOUT_DENSE, LAYOUT_DENSE_CA):
        raise RuntimeError("SdfOracle data file is not dense 0.1.0 layout")
    ca_flag = bool(h["flags"] & FLAG_CONTACT_AWARE)
    if (layout == LAYOUT_DENSE_CA) != ca_flag:
        raise RuntimeError("Dense SDF 0.1.0 contact-aware flag/layout mismatch")
    nx, ny, nz = h["shape"]
    n = nx * ny * nz
    out = dict(layout="dense", spec=dict(bmin=h["bmin"], bmax=h["bmax"], voxel=h["voxel"],
                                         shape=(nx, ny, nz)))
    with open(path, "rb") as f:
        f.seek(128)
        r = _Reader(f, "Failed to read dense SDF payload")
        out["phi"] = r.arr("<f8", n)
        out["normal"] = r.arr("<f8", 3 * n).reshape(n, 3)
        if h["flags"] & FLAG_HESSIAN:
            out["hessian"] = r.arr("<f8", 6 * n).reshape(n, 6)
        else:
            out["hessian"] = np.zeros((n, 6))
        out["witness"] = r.arr("<f8", 3 * n).reshape(n, 3)
        if ca_flag:
            s = _u32(h["reserved"], 4)
            if s <= 0 or s > MAX_CANDIDATES:
                raise RuntimeError("Invalid contact-aware candidate stride")
            cnt = r.arr("<u4", n)
            if np.any(cnt > s):
                raise RuntimeError("Invalid contact-aware candidate count")
            out["ca"] = dict(stride=s, count=cnt.astype(np.uint8), phi=r.arr("<f8", n * s),
                             normal=r.arr("<f8", 3 * n * s).reshape(n * s, 3),
                             branch=r.arr("<i4", n * s))
    return out


def load_sparse(path: str) -> dict:
    """loadSparseSdf (SdfIO.cpp:396-523)."""
    h = read_header(path)
    _check_magic_version(h)
    res = h["reserved"]
    layout = _u32(res, 0)
    ca_flag = bool(h["flags"] & FLAG_CONTACT_AWARE)
    if (layout == LAYOUT_SPARSE_CA) != ca_flag:
        raise RuntimeError("Sparse SDF 0.1.0 contact-aware flag/layout mismatch")
    has_ca = ca_flag and layout == LAYOUT_SPARSE_CA
    if not (h["flags"] & FLAG_SPARSE) or not (layout == LAYOUT_SPARSE or has_ca):
        raise RuntimeError("SdfOracle data file is not sparse block 0.1.0")
    bd = _u32(res, 4)
    halo = _u32(res, 8)
    nblocks = _u32(res, 12)
    band = struct.unpack_from("<d", res, 16)[0]
    stride = _u32(res, 24) if has_ca else 0
    has_h = bool(h["flags"] & FLAG_HESSIAN)
    if bd <= 0 or bd > 1 << 20:
        raise RuntimeError("Sparse SDF blockDim must be positive")
    if has_ca and (stride <= 0 or stride > MAX_CANDIDATES):
        raise RuntimeError("Invalid sparse contact-aware candidate stride")
    V = bd ** 3
    # one block record
    fields = [("hdr", "<i4", (4,)), ("phi", "<f4", (V,)), ("normal", "<f4", (V, 3))]
    if has_h:
        fields.append(("hessian", "<f4", (V, 6)))
    if has_ca:
        fields += [("ca_count", "u1", (V,)), ("ca_phi", "<f4", (V * stride,)),
                   ("ca_normal", "<f4", (V * stride, 3)), ("ca_branch", "<i4", (V * stride,))]
    rec = np.dtype(fields)
    with open(path, "rb") as f:
        f.seek(128)
        b = f.read(rec.itemsize * nblocks)
    full = len(b) // rec.itemsize
    if full < nblocks:
        # distinguish a truncated block header from a truncated payload
        rem = len(b) - full * rec.itemsize
        raise RuntimeError("Failed to read sparse SDF block header" if rem < 16
                           else "Failed to read sparse SDF block payload")
    blocks = np.frombuffer(b, dtype=rec, count=nblocks)
    out = dict(layout="sparse",
               spec=dict(bmin=h["bmin"], bmax=h["bmax"], voxel=h["voxel"], shape=h["shape"]),
               block_dim=bd, halo_voxels=halo, band_distance=band, has_hessian=has_h,
               ijk=np.ascontiguousarray(blocks["hdr"][:, :3]).astype(np.int32),
               phi=np.ascontiguousarray(blocks["phi"]),
               normal=np.ascontiguousarray(blocks["normal"]),
               hessian=np.ascontiguousarray(blocks["hessian"]) if has_h else None)
    if has_ca:
        if np.any(blocks["ca_count"] > stride):
            raise RuntimeError("Invalid sparse contact-aware candidate count")
        out["ca"] = dict(stride=stride, count=np.ascontiguousarray(blocks["ca_count"]),
                         phi=np.ascontiguousarray(blocks["ca_phi"]),
                         normal=np.ascontiguousarray(blocks["ca_normal"]),
                         branch=np.ascontiguousarray(blocks["ca_branch"]))
    return out


def load(path: str) -> dict:
    """SdfOracle::loadFromFile dispatch (SdfOracle.cpp:165-172)."""
    return load_sparse(path) if is_sparse_sdf(path) else load_dense(path)


def save_dense(path: str, spec: dict, phi, normal, hessian=None, witness=None, ca=None) -> bool:
    """saveSdf (SdfIO.cpp:93-183); with ``ca`` (dict stride, count (N,),
    phi (N*s,), normal (N*s,3), branch (N*s,)) the contact-aware dense
    layout 3."""
    n = int(np.prod(spec["shape"]))
    flags = FLAG_HESSIAN | (FLAG_CONTACT_AWARE if ca is not None else 0)
    reserved = (struct.pack("<II", LAYOUT_DENSE_CA, int(ca["stride"])) if ca is not None
                else struct.pack("<I", LAYOUT_DENSE))
    try:
        with open(path, "wb") as f:
            f.write(_header(spec, flags, reserved))
            f.write(np.ascontiguousarray(phi, "<f8").reshape(n).tobytes())
            f.write(np.ascontiguousarray(normal, "<f8").reshape(n, 3).tobytes())
            hs = np.zeros((n, 6)) if hessian is None else hessian
            f.write(np.ascontiguousarray(hs, "<f8").reshape(n, 6).tobytes())
            w = np.zeros((n, 3)) if witness is None else witness
            f.write(np.ascontiguousarray(w, "<f8").reshape(n, 3).tobytes())
            if ca is not None:
                s = int(ca["stride"])
                f.write(np.ascontiguousarray(ca["count"], "<u4").reshape(n).tobytes())
                f.write(np.ascontiguousarray(ca["phi"], "<f8").reshape(n * s).tobytes())
                f.write(np.ascontiguousarray(ca["normal"], "<f8").reshape(n * s, 3).tobytes())
                f.write(np.ascontiguousarray(ca["branch"], "<i4").reshape(n * s).tobytes())
    except OSError:
        return False
    return True


def save_sparse(path: str, spec: dict, block_dim: int, halo_voxels: int, band_distance: float,
                ijk, phi, normal, hessian=None, ca=None) -> bool:
    """saveSparseSdf (SdfIO.cpp:185-275); with ``ca`` (dict stride, count
    (B,V), phi (B,V*s), normal (B,V*s,3), branch (B,V*s)) the contact-aware
    sparse layout 4."""
    if block_dim <= 0:
        return False
    ijk = np.ascontiguousarray(ijk, np.int32).reshape(-1, 3)
    B, V = len(ijk), block_dim ** 3
    flags = (FLAG_SPARSE | (FLAG_HESSIAN if hessian is not None else 0) |
             (FLAG_CONTACT_AWARE if ca is not None else 0))
    reserved = struct.pack("<IIII", LAYOUT_SPARSE_CA if ca is not None else LAYOUT_SPARSE,
                           block_dim, halo_voxels, B) + struct.pack("<d", band_distance)
    if ca is not None:
        reserved += struct.pack("<I", int(ca["stride"]))
    fields = [("hdr", "<i4", (4,)), ("phi", "<f4", (V,)), ("normal", "<f4", (V, 3))]
    if hessian is not None:
        fields.append(("hessian", "<f4", (V, 6)))
    if ca is not None:
        s = int(ca["stride"])
        fields += [("ca_count", "u1", (V,)), ("ca_phi", "<f4", (V * s,)),
                   ("ca_normal", "<f4", (V * s, 3)), ("ca_branch", "<i4", (V * s,))]
    rec = np.zeros(B, dtype=np.dtype(fields))
    rec["hdr"][:, :3] = ijk
    rec["phi"] = np.asarray(phi, np.float32).reshape(B, V)
    rec["normal"] = np.asarray(normal, np.float32).reshape(B, V, 3)
    if hessian is not None:
        rec["hessian"] = np.asarray(hessian, np.float32).reshape(B, V, 6)
    if ca is not None:
        rec["ca_count"] = np.asarray(ca["count"], np.uint8).reshape(B, V)
        rec["ca_phi"] = np.asarray(ca["phi"], np.float32).reshape(B, V * s)
        rec["ca_normal"] = np.asarray(ca["normal"], np.float32).reshape(B, V * s, 3)
        rec["ca_branch"] = np.asarray(ca["branch"], np.int32).reshape(B, V * s)
    try:
        with open(path, "wb") as f:
            f.write(_header(spec, flags, reserved))
            f.write(rec.tobytes())
    except OSError:
        return False
    return True


def load_contact_aware_surface(path: str):
    """loadContactAwareSurfaceFile (SdfSurfaceMesh.cpp:157-344): the
    NEXDYN_CONTACT_AWARE_SURFACE 1 text format -- named surfaces, each with an
    optional row-major 4x4 transform, ``v <id> x y z`` vertices and
    ``tri <id> <v0> <v1> <v2>`` + three corner normals per triangle; normals
    are mapped by the inverse transpose of the transform's linear part and
    normalised.  Returns verts (nv,3), tris (nt,3) int32, corner normals
    (nt,3,3); raises RuntimeError with the reference's messages."""
    def err(line_no, msg):
        return RuntimeError(f"{path}:{line_no}: {msg}")

    def fresh():
        return dict(active=False, name="", nv=-1, nt=-1, sv=0, st=0, T=np.eye(4), N=np.eye(3),
                    ids={})

    def close(line_no, st):
        if not st["active"]:
            return fresh()
        if st["nv"] < 0:
            raise err(line_no, f"surface '{st['name']}' is missing vertices block")
        if st["nt"] < 0:
            raise err(line_no, f"surface '{st['name']}' is missing triangles block")
        if st["sv"] != st["nv"]:
            raise err(line_no, f"surface '{st['name']}' vertex count mismatch")
        if st["st"] != st["nt"]:
            raise err(line_no, f"surface '{st['name']}' triangle count mismatch")
        return fresh()

    try:
        f = open(path, "r")
    except OSError:
        raise RuntimeError(f"Cannot open contact-aware surface file: {path}") from None
    verts, tris, cnorm = [], [], []
    header = False
    st = fresh()
    line_no = 0
    with f:
        for raw in f:
            line_no += 1
            line = raw.split("#", 1)[0].strip()
            if not line:
                continue
            tok = line.split()
            key = tok[0]
            if not header:
                if key != "NEXDYN_CONTACT_AWARE_SURFACE" or len(tok) < 2 or tok[1] != "1":
                    raise err(line_no, "expected header 'NEXDYN_CONTACT_AWARE_SURFACE 1'")
                header = True
                continue
            if key == "surface":
                st = close(line_no, st)
                st["active"] = True
                if len(tok) < 2:
                    raise err(line_no, "surface requires a name")
                st["name"] = tok[1]
                continue
            if key == "end":
                st = close(line_no, st)
                continue
            if not st["active"]:
                raise err(line_no, "expected surface block")
            if key == "transform":
                try:
                    vals = [float(x) for x in tok[1:17]]
                except ValueError:
                    vals = []
                if len(vals) != 16:
                    raise err(line_no, "transform requires 16 row-major values")
                T = np.array(vals).reshape(4, 4)
                L = T[:3, :3]
                if abs(np.linalg.det(L)) <= 1.0e-15:
                    raise err(line_no, "transform linear part must be invertible")
                st["T"] = T
                st["N"] = np.linalg.inv(L).T
                continue
            if key in ("vertices", "triangles"):
                try:
                    cnt = int(tok[1])
                except (IndexError, ValueError):
                    cnt = -1
                if cnt < 0:
                    raise err(line_no, f"{key} requires a non-negative count")
                st["nv" if key == "vertices" else "nt"] = cnt
                continue
            if key == "v":
                if st["nv"] < 0:
                    raise err(line_no, "vertex appears before vertices block")
                try:
                    vid = int(tok[1])
                    p = [float(x) for x in tok[2:5]]
                except (IndexError, ValueError):
                    p = []
                if len(p) != 3:
                    raise err(line_no, "vertex requires: v <id> <x> <y> <z>")
                if vid in st["ids"]:
                    raise err(line_no, "duplicate vertex id in surface")
                st["ids"][vid] = len(verts)
                hp = st["T"] @ np.array([p[0], p[1], p[2], 1.0])
                verts.append(hp[:3] / hp[3] if abs(hp[3]) > 1.0e-15 else hp[:3])
                st["sv"] += 1
                continue
            if key == "tri":
                if st["nt"] < 0:
                    raise err(line_no, "triangle appears before triangles block")
                try:
                    ids = [int(x) for x in tok[2:5]]
                    nums = [float(x) for x in tok[5:14]]
                except (IndexError, ValueError):
                    ids, nums = [], []
                if len(ids) != 3 or len(nums) != 9:
                    raise err(line_no, "triangle requires id, 3 vertex ids, and 3 corner normals")
                nrm = np.array(nums).reshape(3, 3)
                tri = []
                for vid in ids:
                    if vid not in st["ids"]:
                        raise err(line_no, "triangle references unknown vertex id")
                    tri.append(st["ids"][vid])
                out = np.zeros((3, 3))
                for c in range(3):
                    m = st["N"] @ nrm[c]
                    nn = float(np.sqrt(m @ m))
                    if not np.all(np.isfinite(m)) or not np.isfinite(nn) or nn <= 1.0e-15:
                        raise err(line_no, "corner normal must be a finite non-zero vector")
                    out[c] = m / nn
                e0 = verts[tri[1]] - verts[tri[0]]
                e1 = verts[tri[2]] - verts[tri[0]]
                if np.linalg.norm(np.cross(e0, e1)) <= 1.0e-15:
                    raise err(line_no, "triangle is degenerate")
                tris.append(tri)
                cnorm.append(out)
                st["st"] += 1
                continue
            raise err(line_no, f"unknown token '{key}'")
    if not header:
        raise RuntimeError(f"{path}: missing contact-aware surface header")
    close(line_no, st)
    if not verts or not tris:
        raise RuntimeError(f"{path}: contact-aware surface contains no triangles")
    return (np.array(verts, np.float64), np.array(tris, np.int32),
            np.array(cnorm, np.float64).reshape(-1, 3, 3))

"""The C++ plugin API (libsdfo_host.so, headers in host/include/SdfOracle):
SDFO files round-trip byte for byte with files the reference wrote, the
reference's exception messages, and (GPU) SdfBuilder + SdfOracle::queryBatch
against the oracle."""
import os
import subprocess
import sys

import numpy as np
import pytest

from conftest import GOLDEN, PKG, ROOT

CHECK = os.path.join(PKG, "lib", "sdfo_host_check")


@pytest.fixture(scope="module")
def check_bin():
    if not os.path.exists(CHECK):
        subprocess.run([sys.executable, os.path.join(PKG, "build.py")], check=True)
    return CHECK


@pytest.mark.parametrize("name", ["cube8_dense.sdf", "cube16_sparse.sdf", "ca_cube8_dense.sdf",
                                  "ca_cube16_sparse.sdf"])
def test_cpp_io_round_trip_is_byte_exact(check_bin, tmp_path, name):
    src = os.path.join(GOLDEN, name)
    dst = str(tmp_path / name)
    subprocess.run([check_bin, "io", src, dst], check=True)
    assert open(src, "rb").read() == open(dst, "rb").read()


@pytest.mark.parametrize("name", ["cube8_dense.sdf", "cube16_sparse.sdf"])
def test_python_io_round_trip_is_byte_exact(tmp_path, name):
    from sdfo import io as sio

    src = os.path.join(GOLDEN, name)
    d = sio.load(src)
    dst = str(tmp_path / name)
    if d["layout"] == "sparse":
        assert sio.save_sparse(dst, d["spec"], d["block_dim"], d["halo_voxels"],
                               d["band_distance"], d["ijk"], d["phi"], d["normal"], d["hessian"])
    else:
        assert sio.save_dense(dst, d["spec"], d["phi"], d["normal"], d["hessian"], d["witness"])
    assert open(src, "rb").read() == open(dst, "rb").read()
    assert sio.is_valid_sdf(src) and sio.is_sparse_sdf(src) == (d["layout"] == "sparse")


def test_python_io_errors(tmp_path):
    from sdfo import io as sio

    src = open(os.path.join(GOLDEN, "cube8_dense.sdf"), "rb").read()
    bad = tmp_path / "bad.sdf"
    bad.write_bytes(b"XXXX" + src[4:])
    with pytest.raises(RuntimeError, match="Invalid SdfOracle data magic number"):
        sio.load_dense(str(bad))
    bad.write_bytes(src[:4] + (101).to_bytes(4, "little") + src[8:])
    with pytest.raises(RuntimeError, match=r"Unsupported SdfOracle data version: 101 \(only 0.1.0"):
        sio.load_dense(str(bad))
    bad.write_bytes(src[:1000])
    with pytest.raises(RuntimeError, match="Failed to read dense SDF payload"):
        sio.load_dense(str(bad))
    bad.write_bytes(src[:64])
    with pytest.raises(RuntimeError, match="Failed to read SdfOracle data header"):
        sio.load_dense(str(bad))
    with pytest.raises(RuntimeError, match="uses sparse layout; call loadSparseSdf"):
        sio.load_dense(os.path.join(GOLDEN, "cube16_sparse.sdf"))
    with pytest.raises(RuntimeError, match="not sparse block 0.1.0"):
        sio.load_sparse(os.path.join(GOLDEN, "cube8_dense.sdf"))
    with pytest.raises(RuntimeError, match="Cannot open SdfOracle data file"):
        sio.load_dense(str(tmp_path / "missing.sdf"))


def test_python_io_reads_reference_files(port):
    """Arrays read from reference-written files equal the reference build."""
    from sdfo import io as sio
    from sdfo import meshes as M

    d = sio.load(os.path.join(GOLDEN, "cube8_dense.sdf"))
    v, t = M.cube(0.1)
    P = port.build_dense(v, t, padding=0.1, target_resolution=8, max_resolution=8)
    assert np.array_equal(d["phi"], P["phi"]) and np.array_equal(d["normal"], P["normal"])
    assert np.array_equal(d["hessian"], P["hessian"]) and np.array_equal(d["witness"], P["witness"])


def test_cpp_error_messages(check_bin):
    r = subprocess.run([check_bin, "errors"], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.gpu
def test_cpp_build_and_query_batch(cuda, port, check_bin, tmp_path):
    from sdfo import io as sio
    from sdfo import meshes as M

    v, t = M.torus(0.05, 0.01, 48, 12)
    obj = str(tmp_path / "torus.obj")
    M.write_obj(obj, v, t)
    rng = np.random.default_rng(9)
    P = port.build_dense(v, t, padding=0.1, target_resolution=40, max_resolution=40)
    pts = rng.uniform(P["spec"]["bmin"], P["spec"]["bmax"], (3000, 3))
    pts.astype(np.float64).tofile(str(tmp_path / "pts.bin"))
    pre = str(tmp_path / "out")
    r = subprocess.run([check_bin, "build", obj, "40", pre, str(tmp_path / "pts.bin")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    # the OBJ text round trip is exact (%.17g), so the build is the reference's
    d = sio.load_dense(pre + ".dense.sdf")
    for k in ("phi", "normal", "hessian", "witness"):
        assert np.array_equal(d[k], P[k]), k
    Ps = port.build_sparse(v, t, padding=0.1, target_resolution=40, max_resolution=40,
                           band_voxels=3)
    s = sio.load_sparse(pre + ".sparse.sdf")
    assert np.array_equal(s["ijk"], Ps["ijk"]) and np.array_equal(s["phi"], Ps["phi"])
    h = float(P["spec"]["voxel"][0])
    for mode in range(4):
        for layout in ("dense", "sparse"):
            out = np.fromfile(f"{pre}.q{mode}.{layout}.bin").reshape(-1, 8)
            if layout == "dense":
                ref = port.query_dense(P["spec"], P["phi"], P["normal"], P["hessian"], mode, pts)
            else:
                ref = port.query_sparse(Ps["spec"], 8, Ps["ijk"], Ps["phi"], Ps["normal"],
                                        Ps["hessian"], mode, pts)
            valid = out[:, 7] > 0
            assert np.array_equal(valid, ref["valid"])
            assert np.all(np.abs(out[valid, 0] - ref["gap"][valid]) <=
                          1e-5 * np.maximum(np.abs(ref["gap"][valid]), h))


def test_cpp_contact_aware_surface_loader(check_bin, tmp_path):
    """loadContactAwareSurfaceFile of the C++ API against the reference's
    parse of the same file."""
    from conftest import golden

    out = str(tmp_path / "surf.bin")
    subprocess.run([check_bin, "surface", os.path.join(GOLDEN, "torus_small.ncas"), out], check=True)
    raw = np.fromfile(out)
    nv, nt = int(raw[0]), int(raw[1])
    g = golden("torus_small_ncas.npz")
    v = raw[2:2 + 3 * nv].reshape(nv, 3)
    t = raw[2 + 3 * nv:2 + 3 * nv + 3 * nt].reshape(nt, 3).astype(np.int32)
    cn = raw[2 + 3 * nv + 3 * nt:].reshape(nt, 3, 3)
    assert np.array_equal(v, g["verts"]) and np.array_equal(t, g["tris"])
    assert np.allclose(cn, g["corner_normals"], rtol=0, atol=1e-15)


@pytest.mark.gpu
def test_cpp_contact_aware_build_and_queries(cuda, ref, check_bin, tmp_path):
    """SdfBuilder::buildContactAware / buildSparseContactAware of the C++ API
    (GPU) save the reference's bytes; SdfOracle::queryBatch(ContactAware)
    returns the reference's candidate lists."""
    from sdfo import io as sio

    surf = os.path.join(GOLDEN, "torus_small.ncas")
    v, t, cn = ref.load_ca_surface(surf)
    R = ref.build_contact_aware(v, t, cn, target_resolution=24, max_resolution=24)
    Rs = ref.build_contact_aware(v, t, cn, target_resolution=24, max_resolution=24, sparse=True,
                                 band_voxels=3)
    info = R.info()
    rng = np.random.default_rng(4)
    pts = rng.uniform(info["bmin"], info["bmax"], (2000, 3))
    pts.tofile(str(tmp_path / "pts.bin"))
    pre = str(tmp_path / "out")
    r = subprocess.run([check_bin, "ca", surf, "24", pre, str(tmp_path / "pts.bin")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    R.save(str(tmp_path / "ref_dense.sdf"))
    Rs.save(str(tmp_path / "ref_sparse.sdf"))
    assert open(pre + ".ca_dense.sdf", "rb").read() == open(tmp_path / "ref_dense.sdf", "rb").read()
    assert open(pre + ".ca_sparse.sdf", "rb").read() == open(tmp_path / "ref_sparse.sdf", "rb").read()
    h = float(info["voxel"][0])
    for layout, g in (("dense", R), ("sparse", Rs)):
        out = np.fromfile(f"{pre}.ca.{layout}.bin").reshape(-1, 9 + 64)
        q = ref.query_candidates(g, 4, pts)
        v = q["valid"]
        assert np.array_equal(out[:, 7] > 0, v)
        assert np.array_equal(out[v, 8].astype(int), q["ncand"][v])
        assert np.all(np.abs(out[v, 0] - q["gap"][v]) <= 1e-6 * np.maximum(np.abs(q["gap"][v]), h))
        k = out[:, 9:].reshape(-1, 8, 8)
        m = np.arange(8)[None, :] < q["ncand"][:, None]
        assert np.array_equal(k[..., 7][m].astype(np.int64), q["kbranch"][m])
        assert np.all(np.abs(k[..., 0][m] - q["kgap"][m]) <= 1e-6 * np.maximum(np.abs(q["kgap"][m]), h))

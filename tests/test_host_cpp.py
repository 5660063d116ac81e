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


@pytest.mark.parametrize("name", ["cube8_dense.sdf", "cube16_sparse.sdf"])
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

"""SDFO 0.1.0 files straight between disk and device grids
(sdfo_grid_load_file / sdfo_grid_save_file / sdfo_file_probe against
loadSdf / loadSparseSdf / saveSdf / saveSparseSdf / isValidSdf /
isSparseSdf, SdfIO.cpp:93-552).

Error cases are crafted from the golden files; the expected message of each
is pinned against the compiled reference on the CPU (tests without the gpu
marker) and then required of the device loader (gpu tests)."""
import ctypes
import os
import struct

import numpy as np
import pytest

from conftest import GOLDEN

DENSE = os.path.join(GOLDEN, "cube8_dense.sdf")
SPARSE = os.path.join(GOLDEN, "cube16_sparse.sdf")
CA_DENSE = os.path.join(GOLDEN, "ca_cube8_dense.sdf")
CA_SPARSE = os.path.join(GOLDEN, "ca_cube16_sparse.sdf")
FILES = [DENSE, SPARSE, CA_DENSE, CA_SPARSE]


def _read(p):
    with open(p, "rb") as f:
        return bytearray(f.read())


def _put_u32(b, off, v):
    b[off:off + 4] = struct.pack("<I", v)


def _dense_offsets(b):
    """Section offsets of a dense file: phi, n, H, witness, counts, ..."""
    nx, ny, nz = struct.unpack_from("<3I", b, 8)
    N = nx * ny * nz
    o = {"phi": 128, "n": 128 + 8 * N, "H": 128 + 32 * N}
    o["w"] = o["H"] + 48 * N
    o["counts"] = o["w"] + 24 * N
    return N, o


def _sparse_record(b):
    bd = struct.unpack_from("<I", b, 100)[0]
    flags = struct.unpack_from("<I", b, 92)[0]
    layout = struct.unpack_from("<I", b, 96)[0]
    s = struct.unpack_from("<I", b, 120)[0] if layout == 4 else 0
    V = bd ** 3
    off_cnt = 16 + 16 * V + (24 * V if flags & 1 else 0)
    rec = off_cnt + (V + 20 * V * s if s else 0)
    return rec, off_cnt, V


def crafted_cases():
    """(name, bytes, kind) -- kind "any" / "dense" / "sparse"."""
    d, sp, cd, cs = (_read(p) for p in FILES)
    out = []
    out.append(("short_header", d[:100], "any"))
    b = bytearray(d)
    b[0:4] = b"SDFX"
    out.append(("bad_magic", b, "any"))
    b = bytearray(d)
    _put_u32(b, 4, 101)
    out.append(("bad_version", b, "any"))
    out.append(("dense_call_on_sparse", sp, "dense"))
    b = bytearray(d)
    _put_u32(b, 96, 2)
    out.append(("dense_layout_field", b, "dense"))
    b = bytearray(d)
    _put_u32(b, 92, 1 | 4)
    out.append(("dense_ca_flag_without_layout", b, "dense"))
    b = bytearray(cd)
    _put_u32(b, 100, 9)
    out.append(("dense_ca_stride_9", b, "dense"))
    b = bytearray(cd)
    _put_u32(b, 100, 0)
    out.append(("dense_ca_stride_0", b, "dense"))
    N, o = _dense_offsets(d)
    out.append(("dense_cut_in_phi", d[:o["phi"] + 100], "dense"))
    out.append(("dense_cut_in_witness", d[:o["w"] + 8], "dense"))
    out.append(("dense_cut_last_byte", d[:-1], "dense"))
    N, o = _dense_offsets(cd)
    b = bytearray(cd)
    _put_u32(b, o["counts"] + 4 * 37, 5)
    out.append(("dense_ca_count_above_stride", b, "dense"))
    out.append(("dense_ca_bad_count_then_cut", b[:o["counts"] + 4 * 100 + 2], "dense"))
    out.append(("dense_ca_cut_in_counts", cd[:o["counts"] + 4 * 100 + 2], "dense"))
    out.append(("sparse_call_on_dense", d, "sparse"))
    b = bytearray(sp)
    _put_u32(b, 92, 2 | 1 | 4)
    out.append(("sparse_ca_flag_without_layout", b, "sparse"))
    b = bytearray(sp)
    _put_u32(b, 92, 1)
    out.append(("sparse_flag_missing", b, "sparse"))
    b = bytearray(sp)
    _put_u32(b, 100, 0)
    out.append(("sparse_block_dim_0", b, "sparse"))
    b = bytearray(cs)
    _put_u32(b, 120, 0)
    out.append(("sparse_ca_stride_0", b, "sparse"))
    rec, off_cnt, V = _sparse_record(sp)
    out.append(("sparse_cut_in_block_header", sp[:128 + rec + 7], "sparse"))
    out.append(("sparse_cut_at_record_boundary", sp[:128 + 2 * rec], "sparse"))
    out.append(("sparse_cut_in_payload", sp[:128 + 2 * rec + 5000], "sparse"))
    rec, off_cnt, V = _sparse_record(cs)
    b = bytearray(cs)
    b[128 + rec + off_cnt + 11] = 7
    out.append(("sparse_ca_count_above_stride", b, "sparse"))
    out.append(("sparse_ca_bad_count_in_cut_block", b[:128 + rec + off_cnt + 100], "sparse"))
    out.append(("sparse_ca_cut_in_counts", cs[:128 + rec + off_cnt + 100], "sparse"))
    b = bytearray(cs)
    _put_u32(b, 92, 2 | 1)  # sparse CA layout with the CA flag cleared
    out.append(("any_sparse_flag_ca_layout_mismatch", b, "any"))
    b = bytearray(cd)
    _put_u32(b, 92, 2 | 1 | 4)  # dense CA layout with the sparse flag: loadFromFile goes dense
    out.append(("any_dense_layout_sparse_flag", b, "any"))
    return out


# Expected messages, pinned against the compiled reference below.
EXPECTED = {
    "short_header": "Failed to read SdfOracle data header",
    "bad_magic": "Invalid SdfOracle data magic number",
    "bad_version": "Unsupported SdfOracle data version: 101 (only 0.1.0 is supported)",
    "dense_call_on_sparse": "SdfOracle data file uses sparse layout; call loadSparseSdf",
    "dense_layout_field": "SdfOracle data file is not dense 0.1.0 layout",
    "dense_ca_flag_without_layout": "Dense SDF 0.1.0 contact-aware flag/layout mismatch",
    "dense_ca_stride_9": "Invalid contact-aware candidate stride",
    "dense_ca_stride_0": "Invalid contact-aware candidate stride",
    "dense_cut_in_phi": "Failed to read dense SDF payload",
    "dense_cut_in_witness": "Failed to read dense SDF payload",
    "dense_cut_last_byte": "Failed to read dense SDF payload",
    "dense_ca_count_above_stride": "Invalid contact-aware candidate count",
    "dense_ca_bad_count_then_cut": "Invalid contact-aware candidate count",
    "dense_ca_cut_in_counts": "Failed to read dense SDF payload",
    "sparse_call_on_dense": "SdfOracle data file is not sparse block 0.1.0",
    "sparse_ca_flag_without_layout": "Sparse SDF 0.1.0 contact-aware flag/layout mismatch",
    "sparse_flag_missing": "SdfOracle data file is not sparse block 0.1.0",
    "sparse_block_dim_0": "Sparse SDF blockDim must be positive",
    "sparse_ca_stride_0": "Invalid sparse contact-aware candidate stride",
    "sparse_cut_in_block_header": "Failed to read sparse SDF block header",
    "sparse_cut_at_record_boundary": "Failed to read sparse SDF block header",
    "sparse_cut_in_payload": "Failed to read sparse SDF block payload",
    "sparse_ca_count_above_stride": "Invalid sparse contact-aware candidate count",
    "sparse_ca_bad_count_in_cut_block": "Invalid sparse contact-aware candidate count",
    "sparse_ca_cut_in_counts": "Failed to read sparse SDF block payload",
    "any_sparse_flag_ca_layout_mismatch": "Sparse SDF 0.1.0 contact-aware flag/layout mismatch",
    "any_dense_layout_sparse_flag": "SdfOracle data file uses sparse layout; call loadSparseSdf",
}

# Cases the device loader rejects before any device work (header checks).
HEADER_ONLY = {"short_header", "bad_magic", "bad_version", "dense_call_on_sparse",
               "dense_layout_field", "dense_ca_flag_without_layout", "dense_ca_stride_9",
               "dense_ca_stride_0", "sparse_call_on_dense", "sparse_ca_flag_without_layout",
               "sparse_flag_missing", "sparse_block_dim_0", "sparse_ca_stride_0",
               "any_sparse_flag_ca_layout_mismatch", "any_dense_layout_sparse_flag"}


@pytest.fixture(scope="module")
def cases(tmp_path_factory):
    d = tmp_path_factory.mktemp("sdfo_cases")
    out = []
    for name, data, kind in crafted_cases():
        p = str(d / f"{name}.sdf")
        with open(p, "wb") as f:
            f.write(bytes(data))
        out.append((name, p, kind))
    return out


def _lib():
    from sdfo import _native as N

    return N.load()


def _load_error(path, kind):
    from sdfo import _native as N

    out = ctypes.c_void_p()
    rc = _lib().sdfo_grid_load_file(os.fsencode(path), {"any": 0, "dense": 1, "sparse": 2}[kind],
                                    None, ctypes.byref(out))
    if rc == 0:
        _lib().sdfo_grid_destroy(out)
        return rc, None
    return rc, N.last_error()


def test_expected_messages_match_reference(ref, cases):
    assert set(EXPECTED) == {c[0] for c in cases}
    for name, path, kind in cases:
        with pytest.raises(RuntimeError) as e:
            ref.load_kind(path, kind)
        assert str(e.value) == EXPECTED[name], name
    with pytest.raises(RuntimeError) as e:
        ref.load_kind("/nonexistent/x.sdf", "dense")
    assert str(e.value) == "Cannot open SdfOracle data file: /nonexistent/x.sdf"


def test_probe_matches_header_rules(cases):
    from sdfo import io as sio

    lib = _lib()
    v, s = ctypes.c_int32(), ctypes.c_int32()
    paths = FILES + [p for _, p, _ in cases] + ["/nonexistent/x.sdf"]
    for p in paths:
        assert lib.sdfo_file_probe(os.fsencode(p), ctypes.byref(v), ctypes.byref(s)) == 0
        assert bool(v.value) == sio.is_valid_sdf(p), p
        assert bool(s.value) == sio.is_sparse_sdf(p), p
    assert [lib.sdfo_file_probe(os.fsencode(p), ctypes.byref(v), ctypes.byref(s)) or s.value
            for p in FILES] == [0, 1, 0, 1]


def test_header_errors_without_device_work(cases):
    """Header-level rejections happen on the host, with the reference's
    messages, before any CUDA call (so they hold on a machine without a GPU)."""
    from sdfo import _native as N

    for name, path, kind in cases:
        if name not in HEADER_ONLY:
            continue
        rc, msg = _load_error(path, kind)
        assert rc == N.SDFO_ERR_IO and msg == EXPECTED[name], (name, rc, msg)
    rc, msg = _load_error("/nonexistent/x.sdf", "any")
    assert rc == N.SDFO_ERR_IO and msg == "Cannot open SdfOracle data file: /nonexistent/x.sdf"


# --------------------------------------------------------------------- GPU
@pytest.mark.gpu
def test_device_loader_errors_match_reference(cuda, cases):
    from sdfo import _native as N

    for name, path, kind in cases:
        rc, msg = _load_error(path, kind)
        assert rc == N.SDFO_ERR_IO and msg == EXPECTED[name], (name, rc, msg)


@pytest.mark.gpu
@pytest.mark.parametrize("path", FILES, ids=os.path.basename)
def test_load_matches_host_reader_and_save_is_byte_identical(cuda, path, tmp_path):
    from sdfo import SdfGrid
    from sdfo import io as sio

    d = sio.load(path)
    g = SdfGrid.load(path)
    assert g.shape == tuple(d["spec"]["shape"])
    if d["layout"] == "sparse":
        e = g.export_sparse()
        np.testing.assert_array_equal(e["ijk"], d["ijk"])
        np.testing.assert_array_equal(e["phi"], d["phi"])
        np.testing.assert_array_equal(e["normal"], d["normal"])
        if d["hessian"] is not None:
            np.testing.assert_array_equal(e["hessian"], d["hessian"])
        assert (g.block_dim, g.halo_voxels, g.band_distance) == (
            d["block_dim"], d["halo_voxels"], d["band_distance"])
    else:
        e = g.export_dense()
        for k in ("phi", "normal", "hessian", "witness"):
            np.testing.assert_array_equal(e[k], d[k])
    if "ca" in d:
        c = g.export_candidates()
        ca = d["ca"]
        assert c["stride"] == ca["stride"]
        np.testing.assert_array_equal(c["count"], np.asarray(ca["count"]).reshape(-1))
        np.testing.assert_array_equal(c["phi"].reshape(-1), np.asarray(ca["phi"], np.float64).reshape(-1))
        np.testing.assert_array_equal(c["normal"].reshape(-1),
                                      np.asarray(ca["normal"], np.float64).reshape(-1))
        np.testing.assert_array_equal(c["branch"].reshape(-1), np.asarray(ca["branch"]).reshape(-1))
    out = str(tmp_path / "out.sdf")
    assert g.save(out)
    assert _read(out) == _read(path)


@pytest.mark.gpu
def test_queries_identical_after_round_trip(cuda, tmp_path):
    """A device-built dense and sparse grid, saved and loaded back, answer
    every query mode bit for bit as before."""
    import torch

    from sdfo import SdfGrid
    from sdfo import meshes as M

    v, t = M.torus(0.05, 0.015, 64, 24)
    grids = [SdfGrid.build_dense(v, t, target_resolution=48, max_resolution=48),
             SdfGrid.build_sparse(v, t, target_resolution=64, max_resolution=64, band_voxels=3)]
    rng = np.random.default_rng(5)
    pts = torch.tensor(rng.uniform(-0.08, 0.08, (20000, 3)), dtype=torch.float32, device="cuda")
    for i, g in enumerate(grids):
        p = str(tmp_path / f"g{i}.sdf")
        assert g.save(p)
        h = SdfGrid.load(p)
        assert h.is_sparse == g.is_sparse
        for mode in (0, 1, 2, 3):
            a = g.query_tensors(pts, mode=mode, unit=True, witness=True)
            b = h.query_tensors(pts, mode=mode, unit=True, witness=True)
            for k in a:
                assert torch.equal(a[k], b[k]), (i, mode, k)


@pytest.mark.gpu
def test_sparse_save_matches_host_writer(cuda, tmp_path):
    """The device writer's bytes equal the host writer's (sdfo.io.save_sparse,
    itself pinned byte-exact to saveSparseSdf) for a built grid, a grid
    without Hessians and its FP16 re-encoding (written decoded to FP32)."""
    from sdfo import SdfGrid
    from sdfo import io as sio
    from sdfo import meshes as M

    v, t = M.gear_prism(24, 0.05, 0.01, 3000)
    g = SdfGrid.build_sparse(v, t, target_resolution=96, max_resolution=96, band_voxels=3)
    gn = SdfGrid.build_sparse(v, t, target_resolution=96, max_resolution=96, band_voxels=3,
                              store_hessian=False)
    for name, grid in (("h", g), ("noh", gn), ("fp16", g.to_fp16())):
        a = str(tmp_path / f"{name}_dev.sdf")
        b = str(tmp_path / f"{name}_host.sdf")
        assert grid.save(a)
        e = grid.export_sparse()
        sio.save_sparse(b, grid.spec(), grid.block_dim, grid.halo_voxels, grid.band_distance,
                        e["ijk"], e["phi"], e["normal"], e["hessian"])
        assert _read(a) == _read(b), name


@pytest.mark.gpu
def test_save_to_unwritable_path_returns_false(cuda, tmp_path):
    from sdfo import SdfGrid

    g = SdfGrid.load(DENSE)
    assert g.save(str(tmp_path / "no_such_dir" / "x.sdf")) is False

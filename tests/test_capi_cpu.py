"""The C ABI without a GPU: the library loads, exports every function declared
in include/sdfo.h, and its host-only logic (grid setup, argument checks,
error reporting) behaves like the reference's."""
import ctypes
import os
import re

import numpy as np
import pytest

from conftest import ROOT, golden


@pytest.fixture(scope="module")
def lib():
    from sdfo import _native as N

    if not os.path.exists(N.LIB_PATH):
        import subprocess
        import sys

        subprocess.run([sys.executable, os.path.join(ROOT, "sdf-contact-module_b200", "build.py")],
                       check=True)
    return N.load()


def declared_functions():
    src = open(os.path.join(ROOT, "include", "sdfo.h")).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(sdfo_[a-z0-9_]+)\s*\(", src)))


def test_exports_every_declared_symbol(lib):
    names = declared_functions()
    assert len(names) >= 25
    missing = [n for n in names if not hasattr(lib, n)]
    assert not missing, missing


def test_binding_covers_header(lib):
    from sdfo import _native as N

    bound = {n for n, _, _ in N.SIGNATURES}
    assert set(declared_functions()) <= bound


def test_version_and_abi(lib):
    assert lib.sdfo_abi_version() == 1
    assert b"0.1.0" in lib.sdfo_version()


def test_setup_grid_matches_reference(lib):
    """sdfo_setup_grid (host code of the builders) against SdfBuilder::setupGrid
    results recorded from the reference."""
    from sdfo import _native as N
    from sdfo import meshes as M

    g = golden("setup_grid.npz")
    ms = {"cube": M.cube(0.1), "cyl": M.hollow_cylinder(0.05, 0.04, 0.02, n_az=64, n_vert=4),
          "torus": M.torus(0.05, 0.01, 48, 12), "gear": M.gear_prism(24, 0.05, 0.01, 3000)}
    for i, name in enumerate(g["mesh"]):
        v, _ = ms[str(name)]
        v = np.ascontiguousarray(v)
        p = N.BuildParams(float(g["padding"][i]), float(g["voxel_size"][i]), int(g["target"][i]),
                          int(g["maxres"][i]))
        info = N.GridInfo()
        N.check(lib.sdfo_setup_grid(ctypes.c_void_p(v.ctypes.data), len(v), ctypes.byref(p),
                                    ctypes.byref(info)))
        assert tuple(info.shape) == tuple(g["shape"][i])
        assert np.array_equal(np.array(info.bmin[:]), g["bmin"][i])
        assert np.array_equal(np.array(info.bmax[:]), g["bmax"][i])
        assert np.array_equal(np.array(info.voxel[:]), g["voxel"][i])


def test_defaults_match_builder_params(lib):
    from sdfo import _native as N

    p = N.BuildParams()
    lib.sdfo_build_params_default(ctypes.byref(p))
    assert (p.padding, p.voxel_size, p.target_resolution, p.max_resolution) == (0.1, 0.0, 128, 512)
    sp = N.SparseBuildParams()
    lib.sdfo_sparse_build_params_default(ctypes.byref(sp))
    assert (sp.block_dim, sp.halo_voxels, sp.band_voxels, sp.store_hessian, sp.band_distance) == (
        8, 2, 8, 1, 0.0)


def test_empty_mesh_error(lib):
    """SdfBuilder::build throws "Empty mesh provided to SdfBuilder"
    (SdfBuilder.cpp:369-370); the ABI returns SDFO_ERR_EMPTY_MESH with that
    message, before touching the device."""
    from sdfo import _native as N

    p = N.BuildParams(0.1, 0.0, 16, 16)
    out = ctypes.c_void_p()
    v = np.zeros((0, 3))
    rc = lib.sdfo_grid_build_dense(None, 0, None, 0, ctypes.byref(p), None, ctypes.byref(out))
    assert rc == -4
    assert N.last_error() == "Empty mesh provided to SdfBuilder"
    assert out.value is None
    del v


def test_invalid_arguments(lib):
    from sdfo import _native as N

    v = np.ascontiguousarray(np.eye(3))
    t = np.array([[0, 1, 5]], np.int32)
    p = N.BuildParams(0.1, 0.0, 16, 16)
    out = ctypes.c_void_p()
    rc = lib.sdfo_grid_build_dense(ctypes.c_void_p(v.ctypes.data), 3, ctypes.c_void_p(t.ctypes.data),
                                   1, ctypes.byref(p), None, ctypes.byref(out))
    assert rc == -1 and "invalid vertex" in N.last_error()
    sp = N.SparseBuildParams(N.BuildParams(0.1, 0.0, 16, 16), 0, 2, 8, 1, 0.0)
    t = np.array([[0, 1, 2]], np.int32)
    rc = lib.sdfo_grid_build_sparse(ctypes.c_void_p(v.ctypes.data), 3,
                                    ctypes.c_void_p(t.ctypes.data), 1, ctypes.byref(sp), None,
                                    ctypes.byref(out))
    assert rc == -1 and N.last_error() == "Sparse SDF blockDim must be positive"
    bad = np.ascontiguousarray(np.array([[0.0, 0.0, np.nan], [1, 0, 0], [0, 1, 0]]))
    rc = lib.sdfo_grid_build_dense(ctypes.c_void_p(bad.ctypes.data), 3,
                                   ctypes.c_void_p(t.ctypes.data), 1, ctypes.byref(p), None,
                                   ctypes.byref(out))
    assert rc == -1 and "finite" in N.last_error()
    assert lib.sdfo_set_bvh_mode(7) == -1
    assert lib.sdfo_query(None, 3, None, 0, 10, None, None, None, None, None, None, None) == -1
    assert lib.sdfo_grid_destroy(None) == 0


def test_bvh_mode_switch(lib):
    assert lib.sdfo_get_bvh_mode() == 0
    assert lib.sdfo_set_bvh_mode(1) == 0
    assert lib.sdfo_get_bvh_mode() == 1
    assert lib.sdfo_set_bvh_mode(0) == 0


def test_device_check_without_gpu(lib):
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    from sdfo import _native as N

    assert lib.sdfo_device_check(0) == -7
    assert "no CUDA device" in N.last_error()


def test_tuning_round_trip(lib):
    """sdfo_set_tuning / sdfo_get_tuning: host-only state; zero restores a
    field's default; out-of-range values are rejected."""
    from sdfo import _native as N

    before = N.get_tuning()
    try:
        t = N.set_tuning(host_chunk_queries=65536, fill_ctas_per_sm=2, fill_tile_log2_x=2,
                         fill_tile_log2_y=2, host_chunk_growth_pct=150)
        assert t == {"host_chunk_queries": 65536, "fill_ctas_per_sm": 2, "fill_tile_log2_x": 2,
                     "fill_tile_log2_y": 2, "lbvh_traversal": 2, "host_chunk_growth_pct": 150,
                     "host_io_mode": 3, "triangle_cull": 1, "sparse_pair_records": 0,
                     "query_walk": 2}
        assert N.set_tuning(query_walk=1)["query_walk"] == 1
        assert N.set_tuning(query_walk=0)["query_walk"] == 2
        # a rejected tuning applies none of its fields
        bad = N.Tuning(host_chunk_queries=4096, query_walk=3)
        assert lib.sdfo_set_tuning(ctypes.byref(bad)) == -1
        assert N.get_tuning()["host_chunk_queries"] == 65536
        assert N.set_tuning(sparse_pair_records=2)["sparse_pair_records"] == 2
        assert N.set_tuning(sparse_pair_records=1)["sparse_pair_records"] == 1
        assert N.set_tuning(sparse_pair_records=0)["sparse_pair_records"] == 0
        assert N.set_tuning(triangle_cull=2)["triangle_cull"] == 2
        assert N.set_tuning(triangle_cull=0)["triangle_cull"] == 1
        assert N.set_tuning(host_io_mode=3)["host_io_mode"] == 3
        assert N.set_tuning(host_io_mode=1)["host_io_mode"] == 1
        assert N.set_tuning(host_io_mode=0)["host_io_mode"] == 3
        assert N.set_tuning(lbvh_traversal=2)["lbvh_traversal"] == 2
        assert N.set_tuning(lbvh_traversal=1)["lbvh_traversal"] == 1
        assert N.set_tuning(lbvh_traversal=0)["lbvh_traversal"] == 2
        t = N.set_tuning(host_chunk_queries=0, fill_tile_log2_x=0, fill_tile_log2_y=0,
                         host_chunk_growth_pct=0)
        assert t["host_chunk_queries"] == 32768 and t["fill_ctas_per_sm"] == 2
        assert t["host_chunk_growth_pct"] == 130
        bad = N.Tuning(host_chunk_growth_pct=99)
        assert lib.sdfo_set_tuning(ctypes.byref(bad)) == -1
        assert (t["fill_tile_log2_x"], t["fill_tile_log2_y"]) == (3, 3)
        bad = N.Tuning(host_chunk_queries=-1, fill_ctas_per_sm=0)
        assert lib.sdfo_set_tuning(ctypes.byref(bad)) == -1
        bad = N.Tuning(host_chunk_queries=0, fill_ctas_per_sm=65)
        assert lib.sdfo_set_tuning(ctypes.byref(bad)) == -1
        bad = N.Tuning(fill_tile_log2_x=6, fill_tile_log2_y=3)
        assert lib.sdfo_set_tuning(ctypes.byref(bad)) == -1
        assert lib.sdfo_set_tuning(None) == -1
        with pytest.raises(ValueError):
            N.set_tuning(no_such_knob=1)
    finally:
        N.set_tuning(**before)
    assert N.get_tuning() == before


def test_tuning_cache_round_trip(lib, tmp_path):
    """TuningCache stores knobs per (GPU, workload) in JSON and applies the
    sdfo_tuning ones through sdfo_set_tuning."""
    from sdfo import _native as N
    from sdfo.tune import TuningCache, workload_key

    before = N.get_tuning()
    try:
        path = str(tmp_path / "tuning.json")
        c = TuningCache(path)
        key = workload_key("dense_fill", (128, 128, 64), tris=34816)
        assert key == "dense_fill:128x128x64:tris=34816"
        assert c.get("NVIDIA B200", key) is None and not c.apply("NVIDIA B200", key)
        c.put("NVIDIA B200", key, {"fill_tile_log2_x": 2, "fill_tile_log2_y": 2, "threads": 256})
        c2 = TuningCache(path)
        assert c2.get("NVIDIA B200", key)["threads"] == 256
        assert c2.apply("NVIDIA B200", key)
        t = N.get_tuning()
        assert (t["fill_tile_log2_x"], t["fill_tile_log2_y"]) == (2, 2)
        assert c2.get("other GPU", key) is None

        # a batch launch shape goes to the QueryBatch, not to sdfo_set_tuning
        class Batch:
            def __init__(self):
                self.calls = []

            def set_threads(self, t):
                self.calls.append(("threads", t))

            def set_run(self, r):
                self.calls.append(("run", r))

        bkey = workload_key("query_batch", (256,), queries=65536)
        c2.put("NVIDIA B200", bkey, {"threads": 128, "run": 4})
        b = Batch()
        assert TuningCache(path).apply_batch("NVIDIA B200", bkey, b)
        assert b.calls == [("threads", 128), ("run", 4)]
        assert not TuningCache(path).apply_batch("other GPU", bkey, Batch())
        assert not TuningCache(path).apply_batch("NVIDIA B200", key + "x", Batch())
    finally:
        N.set_tuning(**before)

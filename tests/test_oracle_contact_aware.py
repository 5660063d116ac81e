"""Contact-aware builds and queries on the CPU: the oracle restatement
(oracle/sdfo_port.cpp) against fixtures made by the reference itself
(SdfBuilder::buildContactAware / buildSparseContactAware, queryFast in
ContactAware mode, saveSdf / saveSparseSdf, loadContactAwareSurfaceFile;
tests/golden/make_golden.py).  Everything is compared bit for bit."""
import ast
import os

import numpy as np
import pytest

from conftest import GOLDEN, golden

CASES = ["ca_dense_cube", "ca_dense_torus", "ca_sparse_gear", "ca_sparse_cube_notiles"]


def _build(port, g):
    kw = ast.literal_eval(str(g["params"]))
    return port.build_contact_aware(g["verts"], g["tris"], g["corner_normals"], padding=0.1, **kw)


@pytest.mark.parametrize("name", CASES)
def test_port_build_matches_reference(port, name):
    g = golden(f"{name}.npz")
    P = _build(port, g)
    assert tuple(P["spec"]["shape"]) == tuple(g["shape"])
    assert int(P["stride"]) == int(g["stride"])
    for k in ("count", "cphi", "cnormal", "cbranch"):
        assert np.array_equal(P[k], g[k]), k
    if "ijk" in P:
        for k in ("ijk", "phi", "normal", "hessian"):
            assert np.array_equal(P[k], g[f"prim_{k}"]), k
    else:
        for k in ("phi", "normal", "witness", "hessian"):
            assert np.array_equal(P[k], g[f"prim_{k}"]), k
    assert int(g["count"].max()) > 1  # several candidates somewhere


@pytest.mark.parametrize("name", CASES)
def test_port_query_matches_reference(port, name):
    g = golden(f"{name}.npz")
    P = _build(port, g)
    q = port.query_contact_aware(P, g["pts"])
    v = g["q_valid"].astype(bool)
    assert np.array_equal(q["valid"], v)
    assert np.array_equal(q["ncand"][v], g["q_ncand"][v])
    for k in ("gap", "normal", "witness"):
        assert np.array_equal(q[k][v], g[f"q_{k}"][v]), k
    m = np.arange(8)[None, :] < g["q_ncand"][:, None]
    for k in ("kgap", "knormal", "kwitness", "kbranch"):
        assert np.array_equal(q[k][m], g[f"q_{k}"][m]), k
    assert (g["q_ncand"][v] > 1).any()


def test_sdfo_contact_aware_files_round_trip(tmp_path):
    """The reference's contact-aware SDFO files (layouts 3 and 4) load and
    save back byte for byte."""
    from sdfo import io

    d = io.load(os.path.join(GOLDEN, "ca_cube8_dense.sdf"))
    assert d["layout"] == "dense" and d["ca"]["stride"] == 4
    out = tmp_path / "dense.sdf"
    assert io.save_dense(str(out), d["spec"], d["phi"], d["normal"], d["hessian"], d["witness"],
                         ca=d["ca"])
    assert out.read_bytes() == open(os.path.join(GOLDEN, "ca_cube8_dense.sdf"), "rb").read()
    s = io.load(os.path.join(GOLDEN, "ca_cube16_sparse.sdf"))
    assert s["layout"] == "sparse" and s["ca"]["stride"] == 4
    out = tmp_path / "sparse.sdf"
    assert io.save_sparse(str(out), s["spec"], s["block_dim"], s["halo_voxels"],
                          s["band_distance"], s["ijk"], s["phi"], s["normal"], s["hessian"],
                          ca=s["ca"])
    assert out.read_bytes() == open(os.path.join(GOLDEN, "ca_cube16_sparse.sdf"), "rb").read()


def test_contact_aware_surface_loader():
    from sdfo import io

    v, t, cn = io.load_contact_aware_surface(os.path.join(GOLDEN, "torus_small.ncas"))
    g = golden("torus_small_ncas.npz")
    assert np.array_equal(v, g["verts"])
    assert np.array_equal(t, g["tris"])
    assert np.allclose(cn, g["corner_normals"], rtol=0, atol=1e-15)


@pytest.mark.parametrize("text,msg", [
    ("SURFACE 1\n", "expected header"),
    ("NEXDYN_CONTACT_AWARE_SURFACE 1\nv 1 0 0 0\n", "expected surface block"),
    ("NEXDYN_CONTACT_AWARE_SURFACE 1\nsurface a\nvertices 1\nv 1 0 0 0\ntriangles 0\nend\n",
     "contains no triangles"),
    ("NEXDYN_CONTACT_AWARE_SURFACE 1\nsurface a\nvertices 2\nv 1 0 0 0\ntriangles 0\nend\n",
     "vertex count mismatch"),
    ("NEXDYN_CONTACT_AWARE_SURFACE 1\nsurface a\nvertices 3\nv 1 0 0 0\nv 2 1 0 0\nv 3 0 1 0\n"
     "triangles 1\ntri 1 1 2 3 0 0 1 0 0 1 0 0 0\nend\n", "corner normal must be"),
    ("NEXDYN_CONTACT_AWARE_SURFACE 1\nsurface a\nfoo\n", "unknown token 'foo'"),
])
def test_contact_aware_surface_loader_errors(tmp_path, text, msg):
    from sdfo import io

    p = tmp_path / "bad.ncas"
    p.write_text(text)
    with pytest.raises(RuntimeError, match=msg):
        io.load_contact_aware_surface(str(p))

"""Config 5 at full size: perturbed icosphere (subdivision 8, 1,310,720
triangles) as a sparse 512^3 band-3 grid, FP32 and FP16 storage, with
Tricubic queries and their backward.

Gates:
  * build: sparse occupancy, FP32 phi and normal bit-identical to the oracle
    (which replays the reference's tree, so ties resolve alike);
  * FP32 queries: value within 1e-5 * max(|gap|, h), gradient within
    1e-5 * max(|grad|, 1) of the oracle's FP64 interpolation of the same
    payload, on 200k of the 16M benchmark points;
  * FP16 storage: phi is stored as an FP16 fraction of each brick's
    half-range s_b (phi = q * s_b + offset_b), so |d phi| <= 2^-11 s_b, and
    normals as FP16 (|d n| <= 2^-11); the Hermite value weights are bounded
    by 1 in sum of magnitudes (plus the slope weights times h), so a query
    value is within 2^-11 * (s_max + h) + FP32 rounding and the gradient
    within 2^-11 * (3 s_max / h + 3) of the FP64 oracle on the FP32 payload.
    The measured maxima are printed (pytest -s) for the error report;
  * backward: the point gradient against the oracle's gradient and Hessian
    (same bounds as the autograd tests) and the grid-gradient checksums that
    hold at any size -- the value weights of a query sum to 1 (partition of
    unity), so sum(dL/dphi) = sum of dgap over valid queries when dgrad = 0,
    and the derivative weights sum to 0.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu

N_SAMPLE = 200_000


@pytest.fixture(scope="module")
def c5(cuda, port):
    import torch

    from sdfo import SdfGrid
    from sdfo import _native as N
    from sdfo import workloads as W

    c = W.c5_icosphere()
    N.check(N.load().sdfo_set_bvh_mode(N.BVH_REFERENCE))
    grid = SdfGrid.build_sparse(c["verts"], c["tris"], mode=3, **c["sparse"])
    P = port.build_sparse(c["verts"], c["tris"], **c["sparse"])
    h = float(grid.voxel[0])
    pts = W.c5_points(c["verts"], c["tris"], h, n=N_SAMPLE, seed=4)
    torch.cuda.synchronize()
    return c, grid, P, h, pts


def test_c5_build_bit_identical(c5):
    c, grid, P, h, _ = c5
    assert grid.shape == (512, 512, 512)
    assert grid.band_distance == P["band"]
    d = grid.export_sparse()
    assert len(d["ijk"]) > 10_000
    assert np.array_equal(d["ijk"], P["ijk"]), "sparse occupancy"
    assert np.array_equal(d["phi"], P["phi"])
    assert np.array_equal(d["normal"], P["normal"])


def _oracle(port, P, pts):
    return port.query_sparse(P["spec"], P["block_dim"], P["ijk"], P["phi"].astype(np.float64),
                             P["normal"].astype(np.float64), None, 3, pts.astype(np.float64))


def test_c5_fp32_and_fp16_queries_vs_oracle(c5, port):
    import torch

    c, grid, P, h, pts = c5
    ref = _oracle(port, P, pts)
    x = torch.tensor(pts, device="cuda")
    v = ref["valid"]
    assert v.mean() > 0.95
    out = {k: t.cpu().numpy() for k, t in grid.query_tensors(x, mode=3, valid=True).items()}
    assert np.array_equal(out["valid"].astype(bool), v)
    e_gap32 = np.abs(out["gap"] - ref["gap"])[v]
    e_grad32 = np.abs(out["grad"] - ref["grad"])[v]
    assert np.all(e_gap32 <= 1e-5 * np.maximum(np.abs(ref["gap"][v]), h))
    assert np.all(e_grad32 <= 1e-5 * np.maximum(np.abs(ref["grad"][v]), 1.0))

    g16 = grid.to_fp16()
    o16 = {k: t.cpu().numpy() for k, t in g16.query_tensors(x, mode=3, valid=True).items()}
    assert np.array_equal(o16["valid"].astype(bool), v)
    s_max = float(0.5 * (P["phi"].max(axis=1) - P["phi"].min(axis=1)).max())
    e_gap16 = np.abs(o16["gap"] - ref["gap"])[v]
    e_grad16 = np.abs(o16["grad"] - ref["grad"])[v]
    bound_gap = 2.0 ** -11 * (s_max + h) + 1e-5 * h
    bound_grad = 2.0 ** -11 * (3.0 * s_max / h + 3.0)
    print(f"\nC5 error vs FP64 oracle over {int(v.sum())} valid queries (h = {h:.4e} m, "
          f"brick half-range s_max = {s_max / h:.2f} h):\n"
          f"  FP32 storage: max |d gap| = {e_gap32.max() / h:.3e} h, "
          f"max |d grad| = {e_grad32.max():.3e}\n"
          f"  FP16 storage: max |d gap| = {e_gap16.max() / h:.3e} h "
          f"(bound {bound_gap / h:.3e} h), max |d grad| = {e_grad16.max():.3e} "
          f"(bound {bound_grad:.3e})")
    assert e_gap16.max() <= bound_gap
    assert e_grad16.max() <= bound_grad


def test_c5_backward_points_and_grid(c5, port):
    import torch

    c, grid, P, h, pts = c5
    n = len(pts)
    x = torch.tensor(pts, device="cuda")
    rng = np.random.default_rng(8)
    wg = rng.normal(size=n)
    wn = rng.normal(size=(n, 3))
    dgap = torch.tensor(wg, dtype=torch.float32, device="cuda")
    dgrad = torch.tensor(wn, dtype=torch.float32, device="cuda")
    saved = grid.query_linearize(x, mode=3)
    G = torch.zeros((grid.stored_voxels, 4), device="cuda")
    dp = grid.query_backward_saved(x, saved, dgap, dgrad, mode=3, dgrid=G).cpu().numpy()
    ref = _oracle(port, P, pts)
    v = ref["valid"]
    wg32 = dgap.cpu().numpy().astype(np.float64)
    wn32 = dgrad.cpu().numpy().astype(np.float64)
    expect = wg32[:, None] * ref["grad"] + np.einsum("nab,nb->na", ref["hess"], wn32)
    tol = 1e-5 * np.abs(wg32)[:, None] * np.maximum(np.abs(ref["grad"]), 1.0) + \
        2e-5 * np.einsum("nab,nb->na", np.abs(ref["hess"]) + 1.0 / h, np.abs(wn32))
    assert np.all(np.abs(dp[v] - expect[v]) <= tol[v])
    assert np.all(dp[~v] == 0)
    # grid gradient checksums (any size): partition of unity
    ones = torch.ones(n, device="cuda")
    G1 = torch.zeros_like(G)
    grid.query_backward_saved(x, {"valid": saved["valid"]}, ones, None, mode=3, dgrid=G1,
                              want_points=False)
    total = float(G1[:, 0].double().sum())
    assert abs(total - float(v.sum())) <= 1e-4 * float(v.sum())
    for a in range(3):
        e = torch.zeros((n, 3), device="cuda")
        e[:, a] = 1.0
        Ga = torch.zeros_like(G)
        grid.query_backward_saved(x, {"valid": saved["valid"]}, None, e, mode=3, dgrid=Ga,
                                  want_points=False)
        s_phi = float(Ga[:, 0].double().sum())
        s_abs = float(Ga[:, 0].double().abs().sum())
        # derivative weights sum to 0 per query (each is O(1/h)): what is
        # left is FP32 rounding of the weights and of the atomic sums
        assert s_abs > 0.0
        assert abs(s_phi) <= 1e-5 * s_abs

#!/usr/bin/env python
"""Benchmark of the SdfOracle hot path on B200 (one JSON line on rank 0).

Workload (hollow cylinder, R 50 / r 40 / H 20 mm, 512 x 16 segments, 34,816
triangles): dense 128x128x64 FP32 grid and band-3 sparse grid built on the
GPU; 1,000,000 Tricubic value+gradient queries at surface points offset by
N(0, (2h)^2) (seed 1).  One step = one batch of 1M Tricubic queries on the
dense grid with points resident in HBM; L2 is flushed (256 MB write) before
every timed step and each step is timed with CUDA events on its stream.

Also reported (same run, outside the headline loop): sparse-grid queries,
the differentiable query (forward + backward kernels) against the plain
forward query + central finite-difference Jacobian, the fused forward-mode
Jacobian kernel, GPU build throughput (dense, sparse), the ring-on-cube
contact batch with its 6x6 Jacobian against finite differences, the
end-to-end host-buffer path (sdfo_query_host) and the reference's own OpenMP
CPU query loop (oracle/_ref) as the CPU baseline.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Multi-GPU (torchrun): replicas -- every rank runs the full workload on its own
GPU; the step time is the max over ranks (NCCL all-reduce), value = N x
queries / time ("scaling": "weak").
"""
from __future__ import annotations

import argparse
import datetime
import json
import os
import statistics
import subprocess
import sys
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
PKG = os.path.join(ROOT, "sdf-contact-module_b200")
for _p in (ROOT, PKG):
    if _p not in sys.path:
        sys.path.insert(0, _p)

import numpy as np  # noqa: E402

METRIC = "tricubic SDF value+grad queries/s (hollow cylinder 128x128x64 dense FP32, 1M queries)"
WORKLOAD = "hollow_cylinder_r50_r40_h20_512x16_dense128x128x64_1M_tricubic"
N_QUERIES = 1_000_000
TRICUBIC = 3
# algorithmic bytes per Tricubic FP32 query: point 12 + gap 4 + grad 12 +
# valid 1 + 8 corners x {phi, n} 16 B
BYTES_PER_QUERY = 12 + 4 + 12 + 1 + 8 * 16
L2_FLUSH_BYTES = 256 << 20


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    # 2000 headline steps (about 150 ms with the flushes) so that one stall of
    # the device (about 1 ms was seen in single steps) moves the number by
    # about 1 %, not 15 %
    ap.add_argument("--steps", type=int, default=2000)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--kernels-once", choices=["c2", "c4", "c5", "ca", "be", "build", "build5", "contact"],
                    default=None,
                    help="one launch of each query kernel on the workload (for ncu), then exit")
    ap.add_argument("--skip-ca", action="store_true",
                    help="leave out the contact-aware build / query section")
    ap.add_argument("--skip-be", action="store_true",
                    help="leave out the batched Backward-Euler contact step section")
    ap.add_argument("--skip-io", action="store_true",
                    help="leave out the SDFO file load / save section")
    ap.add_argument("--skip-c4", action="store_true",
                    help="leave out the 256-gear batched build / query section")
    ap.add_argument("--skip-c5", action="store_true",
                    help="leave out the 512^3 icosphere section (about 30 s of setup)")
    return ap.parse_args()


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def ncu_traffic(kernel_key):
    """DRAM bytes per launch recorded from an ncu capture (profiles/)."""
    p = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    if not os.path.exists(p):
        return None
    with open(p) as f:
        for line in f:
            parts = line.split()
            if len(parts) >= 2 and parts[0] == kernel_key:
                for kv in parts[1:]:
                    if kv.startswith("dram_bytes_per_launch="):
                        return float(kv.split("=", 1)[1])
    return None


def workload():
    from sdfo import workloads as W

    c = W.c2_cylinder()
    return c


# ---------------------------------------------------------------------------
# clocks during the timed region
# ---------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,utilization.gpu,"
              "clocks_event_reasons.active,clocks_event_reasons.hw_slowdown,"
              "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,"
              "clocks_event_reasons.sw_power_cap")

    def __init__(self, device_index):
        self.proc = None
        self.dev = device_index
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "100", "-i", str(self.dev)], stdout=subprocess.PIPE,
                stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            out, _ = self.proc.communicate(timeout=5)
        except Exception:
            self.proc.kill()
            out, _ = self.proc.communicate()
        rows = []
        for line in out.splitlines():
            f = [x.strip() for x in line.split(",")]
            if len(f) < 10:
                continue
            try:
                rows.append(dict(sm=float(f[1]), max=float(f[2]), util=float(f[4]),
                                 hw=f[6], hwt=f[7], swt=f[8], swp=f[9]))
            except ValueError:
                continue
        if not rows:
            return None
        busy = [r for r in rows if r["util"] > 0] or rows
        reasons = []
        for key, name in (("hw", "hw_slowdown"), ("hwt", "hw_thermal_slowdown"),
                          ("swt", "sw_thermal_slowdown"), ("swp", "sw_power_cap")):
            if any(r[key].lower().startswith("active") for r in busy):
                reasons.append(name)
        return {"sm_mhz": statistics.median(r["sm"] for r in busy),
                "sm_max_mhz": max(r["max"] for r in rows), "reasons": reasons,
                "samples": len(rows), "samples_busy": len([r for r in rows if r["util"] > 0])}


# ---------------------------------------------------------------------------
# reference arm / CPU baseline: the reference's own OpenMP queryFast loop
# ---------------------------------------------------------------------------
def reference_grid(c):
    from oracle import ref

    if ref.available():
        g = ref.build_dense(c["verts"], c["tris"], **c["dense"])
        return g, "reference", ref.max_threads()
    return None, "port", os.cpu_count()


def points_for(c, voxel):
    from sdfo import workloads as W

    return W.c2_points(c["verts"], c["tris"], voxel, N_QUERIES, seed=1)


def cpu_query_rate(c, pts32, repeats):
    """Tricubic queries/s of the reference's OpenMP loop (SdfOracleDemo.cpp:
    373-386 via oracle/_ref), or of the oracle restatement when the compiled
    reference is absent."""
    g, kind, cores = reference_grid(c)
    pts = pts32.astype(np.float64)
    times = []
    if g is not None:
        g.query_bench(TRICUBIC, pts[:1000])
        for _ in range(repeats):
            sec, _, _ = g.query_bench(TRICUBIC, pts)
            times.append(sec)
    else:
        from oracle import port

        P = port.build_dense(c["verts"], c["tris"], **c["dense"])
        for _ in range(repeats):
            t0 = time.perf_counter()
            port.query_dense(P["spec"], P["phi"], P["normal"], None, TRICUBIC, pts)
            times.append(time.perf_counter() - t0)
    return len(pts) * len(times) / sum(times), kind, cores, sum(times)


def cpu_build_rate(c):
    from oracle import ref

    if not ref.available():
        return None
    g = ref.build_dense(c["verts"], c["tris"], **c["dense"])
    n = int(np.prod(g.info()["shape"]))
    return n / g.build_seconds


def run_reference(args, rank, world):
    if rank != 0:
        return
    c = workload()
    from oracle import port

    spec = port.setup_grid(c["verts"], **{k: c["dense"][k] for k in c["dense"]})
    pts = points_for(c, float(spec["voxel"][0])).astype(np.float64)
    g, kind, cores = reference_grid(c)
    if g is None:
        print(json.dumps({"impl": "reference", "unavailable":
                          "compiled reference oracle (oracle/_ref) is not present"}))
        return
    for _ in range(max(args.warmup, 1)):
        g.query_bench(TRICUBIC, pts)
    total = 0.0
    for _ in range(args.steps):
        sec, _, _ = g.query_bench(TRICUBIC, pts)
        total += sec
    value = args.steps * len(pts) / total
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "queries/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1e3 * total / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": WORKLOAD, "queries_per_step": len(pts), "grid": "dense FP64",
                   "l2": "host CPU run"},
        "cpu_baseline": {"value": value, "unit": "queries/s", "cores": cores, "kind": kind,
                         "sample": f"{args.steps} x {len(pts)} Tricubic queryFast calls, "
                                   f"OpenMP static over {cores} threads"},
        "e2e": {"value": value, "unit": "queries/s", "h2d_bytes_per_step": 0,
                "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# our arm
# ---------------------------------------------------------------------------
def timed(torch, fn, steps, warmup, flush, stream, per_step=None):
    """Sum of per-step CUDA-event durations, L2 flushed before each step
    (the durations are appended to per_step when it is a list)."""
    for _ in range(warmup):
        flush()
        fn()
    torch.cuda.synchronize()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
           for _ in range(steps)]
    for s, e in evs:
        flush()
        s.record(stream)
        fn()
        e.record(stream)
    torch.cuda.synchronize()
    ms = [s.elapsed_time(e) for s, e in evs]
    if per_step is not None:
        per_step.extend(ms)
    return sum(ms)


# algorithmic bytes per C5 query (sparse, 8^3 bricks): forward = point 12 +
# gap 4 + grad 12 + valid 1 + 8 corners x {phi, n} (16 B FP32 / 8 B FP16) +
# brick-table entry 4 (+ FP16 per-brick scale/offset 8); the saved-Hessian
# forward adds 24 B (hess6 write).  Backward: dgap 4 + dgrad 12 + grad 12 +
# hess6 24 + dpts 12 (points) and point 12 + valid 1 + table 4 + 8 corners x
# 16 B read-modify-write (grid).
C5_FWD_BYTES = {"fp32": 12 + 4 + 12 + 1 + 8 * 16 + 4, "fp16": 12 + 4 + 12 + 1 + 8 * 8 + 4 + 8}
C5_LIN_EXTRA = 24
C5_BWD_POINTS_BYTES = 4 + 12 + 12 + 24 + 12
C5_BWD_GRID_BYTES = 12 + 1 + 4 + 8 * 16 * 2


def c5_section(torch, lib, N, dev, stream, flush, steps, warmup, peak):
    """Config 5: perturbed icosphere (1.31M tris) sparse 512^3, FP32 and FP16
    storage; 16M Tricubic queries within 4 voxels of the surface; forward,
    differentiable forward + backward w.r.t. points and grid, and the
    forward + central-difference baseline."""
    import ctypes

    from sdfo import SdfGrid
    from sdfo import workloads as W

    def P(t):
        return None if t is None else ctypes.c_void_p(t.data_ptr())

    def sp():
        return ctypes.c_void_p(stream.cuda_stream)

    c = W.c5_icosphere()
    N.check(lib.sdfo_set_bvh_mode(N.BVH_REFERENCE))
    torch.cuda.synchronize()
    # the first build of this size in the process pays one-time costs (the
    # pinned staging block of the host tree, fresh device blocks): timed
    # separately as the cold build, then the build is repeated warm
    t0 = time.perf_counter()
    g_cold = SdfGrid.build_sparse(c["verts"], c["tris"], mode=TRICUBIC, **c["sparse"])
    t_cold = time.perf_counter() - t0
    st_cold = g_cold.build_stats()
    g_cold.close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g32 = SdfGrid.build_sparse(c["verts"], c["tris"], mode=TRICUBIC, **c["sparse"])
    t_build = time.perf_counter() - t0
    st = g32.build_stats()
    N.check(lib.sdfo_set_bvh_mode(N.BVH_LBVH))
    t0 = time.perf_counter()
    gl = SdfGrid.build_sparse(c["verts"], c["tris"], mode=TRICUBIC, **c["sparse"])
    t_lbvh = time.perf_counter() - t0
    st_l = gl.build_stats()
    same_occupancy = bool(gl.block_count == g32.block_count)
    gl.close()
    tuning0 = N.get_tuning()
    N.set_tuning(lbvh_traversal=1)
    gl = SdfGrid.build_sparse(c["verts"], c["tris"], mode=TRICUBIC, **c["sparse"])
    st_stack = gl.build_stats()
    gl.close()
    N.set_tuning(**tuning0)
    N.check(lib.sdfo_set_bvh_mode(N.BVH_REFERENCE))
    # the pseudo-normal sign rule (no parity ray), reference-order tree
    N.check(lib.sdfo_set_sign_mode(N.SIGN_PSEUDONORMAL))
    t0 = time.perf_counter()
    gp = SdfGrid.build_sparse(c["verts"], c["tris"], mode=TRICUBIC, **c["sparse"])
    t_pseudo = time.perf_counter() - t0
    st_p = gp.build_stats()
    gp.close()
    N.check(lib.sdfo_set_sign_mode(N.SIGN_RAY_PARITY))
    g16 = g32.to_fp16()
    h = float(g32.voxel[0])
    pts = torch.tensor(W.c5_points(c["verts"], c["tris"], h), device=dev)
    n = pts.shape[0]
    f32 = dict(device=dev, dtype=torch.float32)
    gap, grad = torch.empty(n, **f32), torch.empty((n, 3), **f32)
    gap16, grad16 = torch.empty(n, **f32), torch.empty((n, 3), **f32)
    valid = torch.empty(n, dtype=torch.uint8, device=dev)
    valid16 = torch.empty(n, dtype=torch.uint8, device=dev)
    hess6 = torch.empty((n, 6), **f32)
    gen = torch.Generator(device=dev).manual_seed(7)
    dgap = torch.randn(n, generator=gen, **f32)
    dgrad = torch.randn((n, 3), generator=gen, **f32)
    dpts = torch.empty((n, 3), **f32)
    dgrid = torch.empty((g32.stored_voxels, 4), **f32)

    def fwd(g, gp, gr, va):
        N.check(lib.sdfo_query(g.handle, TRICUBIC, P(pts), 0, n, P(gp), P(gr), None, None,
                               P(va), None, sp()))

    def ad(g, with_grid):
        N.check(lib.sdfo_query_linearize(g.handle, TRICUBIC, P(pts), n, P(gap), P(grad),
                                         P(valid), P(hess6), sp()))
        if with_grid:
            dgrid.zero_()
        N.check(lib.sdfo_query_backward_saved(g.handle, TRICUBIC, P(pts), n, P(grad), P(hess6),
                                              P(valid), P(dgap), P(dgrad), P(dpts),
                                              P(dgrid) if with_grid else None, sp()))

    fd_h = 1e-3 * h
    shifts = torch.zeros((6, 1, 3), **f32)
    for a in range(3):
        shifts[2 * a, 0, a] = fd_h
        shifts[2 * a + 1, 0, a] = -fd_h
    xfd = torch.empty((6, n, 3), **f32)
    gfd = torch.empty(6 * n, **f32)
    nfd = torch.empty((6 * n, 3), **f32)

    def fd(g):
        fwd(g, gap, grad, valid)
        torch.add(pts.unsqueeze(0), shifts, out=xfd)
        N.check(lib.sdfo_query(g.handle, TRICUBIC, P(xfd), 0, 6 * n, P(gfd), P(nfd), None, None,
                               None, None, sp()))
        gg = gfd.view(3, 2, n)
        nn = nfd.view(3, 2, n, 3)
        return (gg[:, 0] - gg[:, 1]) / (2 * fd_h), (nn[:, 0] - nn[:, 1]) / (2 * fd_h)

    ms = {}
    ms["fwd_fp32"] = timed(torch, lambda: fwd(g32, gap, grad, valid), steps, warmup, flush,
                           stream) / steps
    ms["fwd_fp16"] = timed(torch, lambda: fwd(g16, gap16, grad16, valid16), steps, warmup, flush,
                           stream) / steps
    ms["ad_points_fp32"] = timed(torch, lambda: ad(g32, False), steps, warmup, flush,
                                 stream) / steps
    ms["ad_points_grid_fp32"] = timed(torch, lambda: ad(g32, True), steps, warmup, flush,
                                      stream) / steps
    ms["ad_points_fp16"] = timed(torch, lambda: ad(g16, False), steps, warmup, flush,
                                 stream) / steps
    ms["fd_fp32"] = timed(torch, lambda: fd(g32), steps, warmup, flush, stream) / steps
    # FP16 storage against FP32 storage on the same points (the FP32 grid's
    # own error against the FP64 oracle is pinned by the tests)
    fwd(g32, gap, grad, valid)
    fwd(g16, gap16, grad16, valid16)
    torch.cuda.synchronize()
    both = (valid > 0) & (valid16 > 0)
    dg = (gap16 - gap)[both].abs()
    dn = (grad16 - grad)[both].abs().amax(dim=1)
    gb = C5_FWD_BYTES["fp32"] + C5_LIN_EXTRA + C5_BWD_POINTS_BYTES
    gbg = gb + C5_BWD_GRID_BYTES
    rate = {k: n / (v * 1e-3) for k, v in ms.items()}
    ach = {
        "fwd_fp32": C5_FWD_BYTES["fp32"] * rate["fwd_fp32"] / 1e9,
        "fwd_fp16": C5_FWD_BYTES["fp16"] * rate["fwd_fp16"] / 1e9,
        "ad_points_fp32": gb * rate["ad_points_fp32"] / 1e9,
        "ad_points_grid_fp32": gbg * rate["ad_points_grid_fp32"] / 1e9,
    }
    out = {
        "workload": "perturbed_icosphere_1310720tris_sparse512_band3_16M_tricubic",
        "grid": list(g32.shape), "bricks": g32.block_count, "stored_voxels": g32.stored_voxels,
        "pool_mb_fp32": round(16 * g32.stored_voxels / 2**20, 1),
        "pool_mb_fp16": round(8 * g32.stored_voxels / 2**20, 1),
        "queries_per_step": n, "valid_fraction": float(valid.float().mean()),
        "build_ms": 1e3 * t_build, "build_fill_ms": st["fill_ms"], "build_bvh_ms": st["bvh_ms"],
        "build_setup_ms": st["setup_ms"], "build_hessian_ms": st["hessian_ms"],
        "cold_build_ms": 1e3 * t_cold, "cold_build_bvh_ms": st_cold["bvh_ms"],
        "cold_build_fill_ms": st_cold["fill_ms"], "cold_build_setup_ms": st_cold["setup_ms"],
        "build_stored_voxels_per_s": g32.stored_voxels / t_build,
        "build_candidate_blocks": st["candidate_blocks"],
        "lbvh_build_ms": 1e3 * t_lbvh, "lbvh_fill_ms": st_l["fill_ms"],
        "lbvh_stack_fill_ms": st_stack["fill_ms"],
        "pseudonormal_build_ms": 1e3 * t_pseudo, "pseudonormal_fill_ms": st_p["fill_ms"],
        "pseudonormal_bvh_ms": st_p["bvh_ms"],
        "lbvh_same_block_count": same_occupancy,
        "queries_per_s": rate,
        "ad_vs_fd_speedup_fp32": ms["fd_fp32"] / ms["ad_points_fp32"],
        "gather_model_gbs": ach,
        "hbm_frac": {k: v / peak for k, v in ach.items()},
        "bytes_per_query": {"fwd_fp32": C5_FWD_BYTES["fp32"], "fwd_fp16": C5_FWD_BYTES["fp16"],
                            "ad_points_fp32": gb, "ad_points_grid_fp32": gbg},
        "fp16_vs_fp32": {"max_abs_gap_over_h": float(dg.max()) / h,
                         "mean_abs_gap_over_h": float(dg.mean()) / h,
                         "max_abs_grad": float(dn.max()), "mean_abs_grad": float(dn.mean())},
        "l2": "flushed (256 MB write) before every timed step; brick pool exceeds L2",
    }
    for g in (g16, g32):
        g.close()
    return out


def contact_aware_section(torch, lib, N, dev, stream, flush, steps, warmup, cpu_ok):
    """Contact-aware grids (SdfBuilder::buildContactAware): the hollow
    cylinder with per-face corner normals (sharp rims), dense at the headline
    resolution (128 along the longest axis) and sparse band 3, up to 4
    candidates per voxel; the headline query points in ContactAware mode.
    CPU reference: the reference's contact-aware build of the same mesh at
    resolution 64 (bounded sample)."""
    import ctypes

    from sdfo import SdfGrid
    from sdfo import meshes as M

    c = workload()
    cn = M.corner_normals(c["verts"], c["tris"], "face")
    cv, ct = M.cube(0.1)
    SdfGrid.build_contact_aware(cv, ct, M.corner_normals(cv, ct, "face"), target_resolution=16,
                                max_resolution=16).close()  # warm the kernels
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    g = SdfGrid.build_contact_aware(c["verts"], c["tris"], cn, **c["dense"])
    t_dense = time.perf_counter() - t0
    st = g.build_stats()
    t0 = time.perf_counter()
    gs = SdfGrid.build_contact_aware(c["verts"], c["tris"], cn, sparse=True, band_voxels=3,
                                     **c["dense"])
    t_sparse = time.perf_counter() - t0
    n_vox = int(np.prod(g.shape))
    pts = torch.tensor(points_for(c, float(g.voxel[0])), device=dev)
    n = pts.shape[0]
    gap = torch.empty(n, device=dev)
    grad = torch.empty((n, 3), device=dev)
    valid = torch.empty(n, dtype=torch.uint8, device=dev)

    def P(t):
        return ctypes.c_void_p(t.data_ptr())

    def q(grid):
        N.check(lib.sdfo_query(grid.handle, 4, P(pts), 0, n, P(gap), P(grad), None, None,
                               P(valid), None, ctypes.c_void_p(stream.cuda_stream)))

    q_ms = timed(torch, lambda: q(g), steps, warmup, flush, stream) / steps
    qs_ms = timed(torch, lambda: q(gs), steps, warmup, flush, stream) / steps
    counts = g.export_candidates()["count"]
    out = {
        "workload": "hollow_cylinder_face_normals_ca_dense128x128x64_and_sparse_band3_1M_queries",
        "dense_build_ms": 1e3 * t_dense, "dense_fill_ms": st["fill_ms"],
        "dense_voxels_per_s": n_vox / t_dense,
        "sparse_build_ms": 1e3 * t_sparse, "sparse_stored_voxels_per_s": gs.stored_voxels / t_sparse,
        "mean_candidates": float(counts.mean()), "max_candidates": int(counts.max()),
        "dense_queries_per_s": n / (q_ms * 1e-3), "sparse_queries_per_s": n / (qs_ms * 1e-3),
        "cpu_reference_dense_voxels_per_s": None,
    }
    if cpu_ok:
        from oracle import ref

        if ref.available():
            R = ref.build_contact_aware(c["verts"], c["tris"], cn, target_resolution=64,
                                        max_resolution=64)
            out["cpu_reference_dense_voxels_per_s"] = (
                float(np.prod(R.info()["shape"])) / R.build_seconds)
            out["cpu_reference_sample"] = "buildContactAware of the same mesh at 64^3, OpenMP"
    g.close()
    gs.close()
    return out


def io_section(torch, cpu_ok, repeats=3):
    """SDFO 0.1.0 files straight to and from the device (sdfo_grid_save_file /
    sdfo_grid_load_file) for the headline dense grid (FP64 phi, n, H, witness:
    104 B/voxel) and its sparse band-3 counterpart; wall time of whole calls,
    file in the page cache, median of ``repeats``.  CPU reference: loadSdf /
    saveSdf and loadSparseSdf / saveSparseSdf of the same files."""
    import shutil
    import tempfile

    from sdfo import SdfGrid

    c = workload()
    tmp = tempfile.mkdtemp(prefix="sdfo_io_")
    try:
        out = {"workload": "hollow_cylinder dense 128x128x64 and sparse band 3, SDFO 0.1.0"}
        grids = {"dense": SdfGrid.build_dense(c["verts"], c["tris"], **c["dense"]),
                 "sparse": SdfGrid.build_sparse(c["verts"], c["tris"], **c["sparse"])}
        for name, g in grids.items():
            path = os.path.join(tmp, f"{name}.sdf")
            g.save(path)  # warm: pinned staging, page cache
            SdfGrid.load(path).close()
            save_s, load_s = [], []
            for _ in range(repeats):
                t0 = time.perf_counter()
                assert g.save(path)
                save_s.append(time.perf_counter() - t0)
                t0 = time.perf_counter()
                h = SdfGrid.load(path)
                torch.cuda.synchronize()
                load_s.append(time.perf_counter() - t0)
                st = h.build_stats()
                h.close()
            size = os.path.getsize(path)
            out[name] = {"file_bytes": size, "save_ms": 1e3 * statistics.median(save_s),
                         "load_ms": 1e3 * statistics.median(load_s),
                         "save_gbs": size / statistics.median(save_s) / 1e9,
                         "load_gbs": size / statistics.median(load_s) / 1e9,
                         "last_load_phases_ms": {"allocate": st["setup_ms"],
                                                 "read_and_transfer": st["fill_ms"],
                                                 "decode": st["hessian_ms"]}}
            if cpu_ok:
                from oracle import ref

                if ref.available():
                    rl, rs = [], []
                    for _ in range(repeats):
                        R = ref.load_kind(path, name)
                        rl.append(R.build_seconds)
                        ok, sec = ref.save_timed(R, os.path.join(tmp, f"{name}_ref.sdf"))
                        rs.append(sec)
                        del R
                    out[name]["cpu_reference_load_ms"] = 1e3 * statistics.median(rl)
                    out[name]["cpu_reference_save_ms"] = 1e3 * statistics.median(rs)
            g.close()
        return out
    finally:
        shutil.rmtree(tmp, ignore_errors=True)


def be_section(torch, dev, stream, steps, warmup, cpu_ok):
    """Batched BackwardEulerIntegrator.step on the GPU (sdfo.be.BEStepper):
    2048 ring drops on a slab (7,680 quadrature points each), `steps`
    consecutive steps of dt = 1 ms from the drop (free flight with the
    time-of-impact search, impact, contact at 10 us steps), each step one
    launch for all scenes, timed with CUDA events.  CPU baseline: the NumPy
    restatement of the reference integrator (oracle/be_port.py, which follows
    implicit_be.py operation for operation) on the first scenes."""
    from sdfo import SdfGrid
    from sdfo import workloads as W
    from sdfo.be import BEStepper, default_params

    c = W.be_ring_drops(2048)
    grid = SdfGrid.build_dense(*c["slab"], **c["build"])
    p = c["params"]

    def stepper(tangent):
        return BEStepper(grid, c["quad_x"], c["quad_w"], c["mass"], c["inertia"], p["stiffness"],
                         order=p["order"], damping=p["damping"], friction=p["friction"],
                         regularizer=p["regularizer"], activation_distance=p["activation_distance"],
                         narrow_margin=0.01, max_scenes=len(c["r"]),
                         params=default_params(tangent=tangent))

    def run(st):
        warm = st.scenes(c["r"], c["R"], c["v"], c["w"])
        for _ in range(max(1, warmup)):
            st.step(warm, 1e-3)
        scenes = st.scenes(c["r"], c["R"], c["v"], c["w"])
        torch.cuda.synchronize()
        st.stats(reset=True)
        evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
               for _ in range(steps)]
        for a, b in evs:
            a.record(stream)
            st.step(scenes, 1e-3, stream=stream)
            b.record(stream)
        torch.cuda.synchronize()
        return scenes, [a.elapsed_time(b) for a, b in evs], st.stats()

    # the exact-Newton mode (exact contact every residual, analytic tangent)
    st_ex = stepper("exact")
    scenes_ex, ms_ex, stats_ex = run(st_ex)
    u_ex = st_ex.unpack(scenes_ex)
    st_ex.close()
    st = stepper("reference")
    scenes, ms, stats_ref = run(st)
    graph_scenes = st.scenes(c["r"], c["R"], c["v"], c["w"])
    torch.cuda.synchronize()
    # the same steps as integrate runs them: one CUDA graph of `steps`
    # launches (t_end far enough that every step is the full 1 ms request)
    start = graph_scenes.clone()
    t_end = graph_scenes[:, 18] + 1.0
    st.advance(graph_scenes, t_end, 1e-3, launches=steps, stream=stream)  # captured here (untimed)
    torch.cuda.synchronize()
    graph_scenes.copy_(start)
    ga, gb = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    ga.record(stream)
    st.advance(graph_scenes, t_end, 1e-3, launches=steps, stream=stream)
    gb.record(stream)
    torch.cuda.synchronize()
    u = st.unpack(scenes)
    n = len(c["r"])
    same_t = u["t"] == u_ex["t"]
    dr = np.abs(u["r"] - u_ex["r"]).max(axis=1)[same_t]
    out = {"workload": "ring_drops_on_slab_2048_scenes_7680_points_dt1ms",
           "scenes": n, "steps": steps, "step_ms": ms,
           "scene_steps_per_s": n * steps / (sum(ms) * 1e-3),
           "tangent": "reference (linearisation cache + heuristic diagonal tangent)",
           "newton_iterations": stats_ref["newton_iterations"],
           "residual_evaluations": stats_ref["residual_evaluations"],
           "be_solves": stats_ref["be_solves"],
           "newton_per_solve": stats_ref["newton_iterations"] / max(1, stats_ref["be_solves"]),
           "exact": {"tangent": "exact contact every residual + analytic dR/dV",
                     "step_ms": ms_ex, "scene_steps_per_s": n * steps / (sum(ms_ex) * 1e-3),
                     "newton_iterations": stats_ex["newton_iterations"],
                     "residual_evaluations": stats_ex["residual_evaluations"],
                     "be_solves": stats_ex["be_solves"],
                     "newton_per_solve": stats_ex["newton_iterations"] / max(1, stats_ex["be_solves"]),
                     "scenes_same_time_as_reference": int(same_t.sum()),
                     "max_abs_dr_vs_reference_m": float(dr.max()) if dr.size else None,
                     "phases_after": {str(k): int((u_ex["phase"] == k).sum())
                                      for k in sorted(set(u_ex["phase"].tolist()))}},
           "graph_ms": ga.elapsed_time(gb),
           "graph_matches_steps": bool(torch.equal(graph_scenes, scenes)),
           "simulated_time_per_scene_s": float(u["t"].mean()),
           "phases_after": {str(k): int((u["phase"] == k).sum()) for k in sorted(set(u["phase"].tolist()))},
           "cpu_port_scene_steps_per_s": None}
    if cpu_ok:
        from oracle import be_port as P

        g64 = grid.export_dense()
        spec = dict(bmin=grid.bmin, voxel=grid.voxel, shape=grid.shape)
        from oracle import interp_np

        def qb(Y):
            gap, grad, valid, _ = interp_np.query(spec, g64["phi"], g64["normal"], 2, Y)
            gn = np.linalg.norm(grad, axis=1)
            unit = np.zeros_like(grad)
            unit[:, 2] = 1.0
            ok = valid & (gn > 1e-30)
            unit[ok] = grad[ok] / gn[ok, None]
            return gap, grad, gn, unit, valid

        w = c["quad_w"] / c["quad_w"].sum()
        sc = P.Scene(qb, c["quad_x"], w, grid.bmin, grid.bmax, 0.01, p["stiffness"], p["order"],
                     p["damping"], p["friction"], p["regularizer"], c["mass"], c["inertia"])
        t0 = time.perf_counter()
        done = 0
        for i in range(4):
            integ = P.Integrator(sc)
            s = P.BodyState(c["r"][i].copy(), c["R"][i].copy(), c["v"][i].copy(), c["w"][i].copy())
            for _ in range(steps):
                integ.step(s, 1e-3)
                done += 1
            if time.perf_counter() - t0 > 20.0:
                break
        out["cpu_port_scene_steps_per_s"] = done / (time.perf_counter() - t0)
        out["cpu_port_sample"] = f"{done} scene-steps of the first scenes, one host thread (NumPy)"
    st.close()
    return out


# algorithmic bytes per C4 query (posed, batched, sparse 8^3 bricks): point
# 12 + gap 4 + grad 12 + valid 1 + 8 corners x {phi, n} 16 B + brick-table
# entry 4 (the per-grid pose, 96 B per 65,536 queries, is left out)
C4_BYTES_PER_QUERY = 12 + 4 + 12 + 1 + 8 * 16 + 4


def c4_section(torch, lib, N, dev, stream, flush, steps, warmup, peak):
    """Config 4: 256 gear prisms (2k-60k tris, sparse 64^3..256^3, band 3):
    one batched build against 256 single builds, then 256 x 65,536 Tricubic
    queries under random poses as one captured CUDA graph (the launch shape
    picked by the autotuner) against 256 per-grid launches."""
    from sdfo import SdfGrid
    from sdfo import workloads as W
    from sdfo.batch import QueryBatch, pack_poses
    from sdfo.tune import tune_query_batch

    gears = W.c4_gears()
    args = [dict(verts=g["verts"], tris=g["tris"], **g["sparse"]) for g in gears]
    N.check(lib.sdfo_set_bvh_mode(N.BVH_REFERENCE))
    for g in SdfGrid.build_sparse_batched(args[:8]):  # warm
        g.close()
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    grids = SdfGrid.build_sparse_batched(args, mode=TRICUBIC)
    t_batch = time.perf_counter() - t0
    st = grids[0].build_stats()
    t0 = time.perf_counter()
    for a in args:
        SdfGrid.build_sparse(a["verts"], a["tris"], mode=TRICUBIC,
                             **{k: v for k, v in a.items() if k not in ("verts", "tris")}).close()
    torch.cuda.synchronize()
    t_single = time.perf_counter() - t0
    stored = sum(g.stored_voxels for g in grids)
    n_per = 65_536
    rng = np.random.default_rng(3)
    world, R, t = [], [], []
    for g, grid in zip(gears, grids):
        p = W.near_surface_points(g["verts"], g["tris"], float(grid.voxel[0]), n_per,
                                  int(rng.integers(1 << 30)))
        k = rng.normal(size=3)
        k /= np.linalg.norm(k)
        ang = rng.uniform(0.0, np.pi)
        K = np.array([[0.0, -k[2], k[1]], [k[2], 0.0, -k[0]], [-k[1], k[0], 0.0]])
        Rg = np.eye(3) + np.sin(ang) * K + (1.0 - np.cos(ang)) * (K @ K)
        tg = rng.uniform(-0.5, 0.5, 3)
        world.append((p.astype(np.float64) @ Rg.T + tg).astype(np.float32))
        R.append(Rg)
        t.append(tg)
    x = torch.tensor(np.concatenate(world), device=dev)
    poses = pack_poses(np.array(R), np.array(t), device=dev)
    qb = QueryBatch(grids, [n_per] * len(grids))
    tuned = tune_query_batch(qb, x, poses, reps=10, warmup=2)
    graph, out = qb.capture(x, poses)
    total = qb.total
    graph_ms = timed(torch, graph.replay, steps, warmup, flush, stream) / steps
    # the same queries as 256 separate single-grid launches (local points)
    import ctypes

    xs = [x[i * n_per:(i + 1) * n_per] for i in range(len(grids))]
    gap = torch.empty(n_per, device=dev)
    grad = torch.empty((n_per, 3), device=dev)

    def per_grid():
        for grid, xi in zip(grids, xs):
            N.check(lib.sdfo_query(grid.handle, TRICUBIC, ctypes.c_void_p(xi.data_ptr()), 0, n_per,
                                   ctypes.c_void_p(gap.data_ptr()), ctypes.c_void_p(grad.data_ptr()),
                                   None, None, None, None, ctypes.c_void_p(stream.cuda_stream)))

    per_grid_ms = timed(torch, per_grid, max(3, steps // 4), warmup, flush, stream) / max(3, steps // 4)
    valid = float(out[2].float().mean())
    graph_rate = total / (graph_ms * 1e-3)
    res = {
        "workload": "256_gear_prisms_sparse64-256_band3_65536q_each_tricubic_posed",
        "meshes": len(grids), "triangles": int(sum(len(g["tris"]) for g in gears)),
        "stored_voxels": int(stored), "bricks": int(sum(g.block_count for g in grids)),
        "batched_build_ms": 1e3 * t_batch, "single_builds_ms": 1e3 * t_single,
        "batched_build_speedup": t_single / t_batch,
        "batched_fill_ms": st["fill_ms"], "batched_bvh_ms": st["bvh_ms"],
        "batched_stored_voxels_per_s": stored / t_batch,
        "queries": total, "valid_fraction": valid,
        "graph_queries_per_s": graph_rate,
        "bytes_per_query": C4_BYTES_PER_QUERY,
        "gather_model_gbs": C4_BYTES_PER_QUERY * graph_rate / 1e9,
        "hbm_frac": C4_BYTES_PER_QUERY * graph_rate / 1e9 / peak,
        "pool_mb": round(16 * stored / 2**20, 1),
        "per_grid_launches_queries_per_s": total / (per_grid_ms * 1e-3),
        "graph_vs_per_grid_speedup": per_grid_ms / graph_ms,
        "autotuned_threads": tuned["threads"],
        "autotuned_run_tiles": tuned["run"],
        "autotune_ms": {str(k): v for k, v in tuned["ms"].items()},
    }
    qb.close()
    for g in grids:
        g.close()
    return res


def run_ours(args, rank, world, local_rank):
    import torch

    import sdfo
    from sdfo import SdfGrid
    from sdfo import _native as N
    from sdfo.contact import ContactBatch, fd_jacobian, pack_states
    from sdfo import workloads as W

    torch.cuda.set_device(local_rank)
    N.check(N.load().sdfo_device_check(local_rank))
    dev = torch.device("cuda", local_rank)
    stream = torch.cuda.current_stream()
    lib = N.load()
    c = workload()
    clocks = ClockSampler(local_rank)
    clocks.start()

    # ---- builds (reference-order BVH: bit-identical to the reference) ----
    N.check(lib.sdfo_set_bvh_mode(N.BVH_REFERENCE))
    SdfGrid.build_dense(c["verts"], c["tris"], **c["dense"]).close()  # warm
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    dense = SdfGrid.build_dense(c["verts"], c["tris"], mode=TRICUBIC, **c["dense"])
    t_dense = time.perf_counter() - t0
    st_dense = dense.build_stats()
    t0 = time.perf_counter()
    sparse = SdfGrid.build_sparse(c["verts"], c["tris"], mode=TRICUBIC, **c["sparse"])
    t_sparse = time.perf_counter() - t0
    st_sparse = sparse.build_stats()
    N.check(lib.sdfo_set_bvh_mode(N.BVH_LBVH))
    SdfGrid.build_dense(c["verts"], c["tris"], **c["dense"]).close()
    t0 = time.perf_counter()
    lb = SdfGrid.build_dense(c["verts"], c["tris"], **c["dense"])
    t_lbvh = time.perf_counter() - t0
    st_lbvh = lb.build_stats()
    lb.close()
    N.check(lib.sdfo_set_bvh_mode(N.BVH_REFERENCE))
    n_vox = int(np.prod(dense.shape))
    # build knobs on this box (each result bit-identical, per the tests):
    # the FP32 triangle cull on/off, the LBVH walk with a stack or stackless
    knobs = {}
    tuning0 = N.get_tuning()

    def fill_ms(kind, **kw):
        out = []
        for _ in range(3):
            g = (SdfGrid.build_dense if kind == "dense" else SdfGrid.build_sparse)(
                c["verts"], c["tris"], **(c["dense"] if kind == "dense" else c["sparse"]))
            out.append(g.build_stats()["fill_ms"])
            g.close()
        return float(np.median(out))

    for cull in (1, 2):
        N.set_tuning(triangle_cull=cull)
        key = "cull_on" if cull == 1 else "cull_off"
        knobs[key] = {"dense_fill_ms": fill_ms("dense"), "sparse_fill_ms": fill_ms("sparse")}
    N.set_tuning(**tuning0)
    N.check(lib.sdfo_set_bvh_mode(N.BVH_LBVH))
    for trav in (1, 2):
        N.set_tuning(lbvh_traversal=trav)
        knobs["lbvh_stack" if trav == 1 else "lbvh_stackless"] = {"dense_fill_ms": fill_ms("dense")}
    N.set_tuning(**tuning0)
    N.check(lib.sdfo_set_bvh_mode(N.BVH_REFERENCE))
    # traversal work per voxel of the dense fill (instrumented copy, untimed)
    trav = SdfGrid.traversal_stats(c["verts"], c["tris"], **c["dense"])
    trav.pop("totals")

    h = float(dense.voxel[0])
    pts_np = points_for(c, h)
    pts = torch.tensor(pts_np, device=dev)
    n = pts.shape[0]
    flush_buf = torch.empty(L2_FLUSH_BYTES // 4, dtype=torch.float32, device=dev)

    def flush():
        flush_buf.zero_()

    import ctypes

    gap = torch.empty(n, device=dev)
    grad = torch.empty((n, 3), device=dev)
    valid = torch.empty(n, dtype=torch.uint8, device=dev)

    def P(t):
        return None if t is None else ctypes.c_void_p(t.data_ptr())

    def sptr():
        return ctypes.c_void_p(stream.cuda_stream)

    def launch(grid, x, g_out, n_out, v_out=None, h_out=None, m=TRICUBIC):
        N.check(lib.sdfo_query(grid.handle, m, P(x), 0, x.shape[0], P(g_out), P(n_out), None,
                               None, P(v_out), P(h_out), sptr()))

    def query(grid, out_hess=None):
        launch(grid, pts, gap, grad, valid, out_hess)

    # ---- headline: dense Tricubic forward ----
    if world > 1:
        torch.distributed.barrier()
    torch.cuda.synchronize()
    head_steps = []
    total_ms = timed(torch, lambda: query(dense), args.steps, args.warmup, flush, stream, head_steps)
    t_local = torch.tensor([total_ms], dtype=torch.float64, device=dev)
    if world > 1:
        torch.distributed.barrier()
        torch.distributed.all_reduce(t_local, op=torch.distributed.ReduceOp.MAX)
    total_ms_max = float(t_local.item())
    ms_step = total_ms_max / args.steps
    value = world * args.steps * n / (total_ms_max * 1e-3)
    per_launch_s = (total_ms / args.steps) * 1e-3

    # ---- sparse grid forward ----
    sparse_ms = timed(torch, lambda: query(sparse), args.steps, args.warmup, flush, stream) / args.steps

    # ---- differentiable query: forward + backward (VJP) kernels ----
    dgap = torch.randn(n, device=dev)
    dgrad = torch.randn((n, 3), device=dev)
    dpts = torch.empty((n, 3), device=dev)

    hess6 = torch.empty((n, 6), device=dev)

    def ad_step():
        # what sdfo.autograd runs for float32 points: forward + saved Hessian,
        # then the elementwise backward (no second stencil gather)
        N.check(lib.sdfo_query_linearize(dense.handle, TRICUBIC, P(pts), n, P(gap), P(grad),
                                         P(valid), P(hess6), sptr()))
        N.check(lib.sdfo_query_backward_saved(dense.handle, TRICUBIC, P(pts), n, P(grad),
                                              P(hess6), P(valid), P(dgap), P(dgrad), P(dpts),
                                              None, sptr()))

    def ad_regather_step():
        query(dense)
        N.check(lib.sdfo_query_backward(dense.handle, TRICUBIC, P(pts), n, P(dgap), P(dgrad),
                                        P(dpts), None, sptr()))

    ad_ms = timed(torch, ad_step, args.steps, args.warmup, flush, stream) / args.steps
    ad_rg_ms = timed(torch, ad_regather_step, args.steps, args.warmup, flush, stream) / args.steps
    hess = torch.empty((n, 3, 3), device=dev)
    jac_ms = timed(torch, lambda: query(dense, out_hess=hess), args.steps, args.warmup, flush,
                   stream) / args.steps
    # plain forward + central finite differences (6 shifted copies of the batch)
    fd_h = 1e-3 * h
    shifts = torch.zeros((6, 1, 3), device=dev)
    for a in range(3):
        shifts[2 * a, 0, a] = fd_h
        shifts[2 * a + 1, 0, a] = -fd_h
    xfd = torch.empty((6, n, 3), device=dev)
    gfd = torch.empty(6 * n, device=dev)
    nfd = torch.empty((6 * n, 3), device=dev)

    def fd_step():
        query(dense)
        torch.add(pts.unsqueeze(0), shifts, out=xfd)
        launch(dense, xfd.view(-1, 3), gfd, nfd)
        gg = gfd.view(3, 2, n)
        nn = nfd.view(3, 2, n, 3)
        dg = (gg[:, 0] - gg[:, 1]) / (2 * fd_h)        # d gap / d x_a
        dn = (nn[:, 0] - nn[:, 1]) / (2 * fd_h)        # d grad / d x_a
        return dg, dn

    fd_ms = timed(torch, fd_step, args.steps, args.warmup, flush, stream) / args.steps

    # ---- end-to-end through the C ABI with host buffers ----
    hp = torch.from_numpy(pts_np).pin_memory()
    hg = torch.empty(n, dtype=torch.float32).pin_memory()
    hn = torch.empty((n, 3), dtype=torch.float32).pin_memory()
    hv = torch.empty(n, dtype=torch.uint8).pin_memory()

    def e2e_step():
        N.check(lib.sdfo_query_host(dense.handle, TRICUBIC, P(hp), 0, n, P(hg), P(hn), None, None,
                                    P(hv), sptr()))

    for _ in range(args.warmup):
        e2e_step()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    e2e_s = time.perf_counter() - t0
    e2e_value = args.steps * n / e2e_s
    if world > 1:
        e = torch.tensor([e2e_s], dtype=torch.float64, device=dev)
        torch.distributed.all_reduce(e, op=torch.distributed.ReduceOp.MAX)
        e2e_value = world * args.steps * n / float(e.item())
    # the same call with each host io mode (sdfo_tuning.host_io_mode): staged
    # copies per growing chunk, results written in place, both ways in place
    tuning0 = N.get_tuning()
    e2e_modes = {}
    for name, io in (("staged_copies", 1), ("results_in_place", 2), ("zero_copy", 3)):
        N.set_tuning(host_io_mode=io)
        for _ in range(args.warmup):
            e2e_step()
        reps = max(20, min(args.steps, 200))
        t0 = time.perf_counter()
        for _ in range(reps):
            e2e_step()
        e2e_modes[name] = reps * n / (time.perf_counter() - t0)
    N.set_tuning(**tuning0)

    # ---- contact: ring on cube, 4096 poses, forward + 6x6 Jacobian ----
    cc = W.c3_ring_cube(n_poses=4096)
    cube = SdfGrid.build_dense(*cc["cube"], **cc["build"])
    batch = ContactBatch(cube, cc["quad_x"], cc["quad_w"], mode=2, **cc["params"])
    poses = pack_states(cc["r"], cc["R"], cc["v"], cc["w"], device=dev)
    body_b = pack_states(np.zeros((1, 3)), np.eye(3)[None], device=dev)[0]
    csteps = max(3, args.steps // 20)
    ct_ad = timed(torch, lambda: batch.evaluate(poses, body_b, jacobian=True), csteps,
                  args.warmup, flush, stream) / csteps
    ct_fwd = timed(torch, lambda: batch.evaluate(poses, body_b), csteps, args.warmup, flush,
                   stream) / csteps
    ct_fd = timed(torch, lambda: fd_jacobian(batch, poses, body_b), csteps, args.warmup, flush,
                  stream) / csteps
    batch3 = ContactBatch(cube, cc["quad_x"], cc["quad_w"], mode=3, **cc["params"])
    ct_ad3 = timed(torch, lambda: batch3.evaluate(poses, body_b, jacobian=True), csteps,
                   args.warmup, flush, stream) / csteps
    peak, peak_src = measured_peaks()
    ca = None
    if not args.skip_ca:
        ca = contact_aware_section(torch, lib, N, dev, stream, flush, max(3, args.steps // 10),
                                   args.warmup, rank == 0 and world == 1)
    be_out = None
    if not args.skip_be:
        be_out = be_section(torch, dev, stream, 10, 1, rank == 0 and world == 1)
    sdfo_io = None
    if not args.skip_io:
        sdfo_io = io_section(torch, rank == 0 and world == 1)
    c4 = None
    if not args.skip_c4:
        c4 = c4_section(torch, lib, N, dev, stream, flush, max(3, args.steps // 20), args.warmup,
                        peak)
    c5 = None
    if not args.skip_c5:
        c5 = c5_section(torch, lib, N, dev, stream, flush, max(3, args.steps // 20),
                        args.warmup, peak)
    clk = clocks.stop()

    # ---- CPU baseline (reference OpenMP loop), rank 0 only ----
    cpu = None
    cpu_build = None
    if rank == 0 and world == 1:
        rate, kind, cores, secs = cpu_query_rate(c, pts_np, repeats=3)
        cpu = {"value": rate, "unit": "queries/s", "cores": cores, "kind": kind,
               "sample": f"3 x {n} Tricubic queryFast calls on the same points, OpenMP static "
                         f"({secs:.2f} s of CPU time)"}
        cpu_build = cpu_build_rate(c)

    achieved = BYTES_PER_QUERY * n / per_launch_s / 1e9
    walk = N.get_tuning()["query_walk"] == 2
    head_kernel = "k_query_walk<Tricubic,dense>" if walk else "k_query_pipe<Tricubic,dense>"
    traffic = ncu_traffic("tricubic_dense_c2_walk" if walk else "tricubic_dense_c2")
    line = {
        "metric": METRIC, "value": value, "unit": "queries/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_step,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": WORKLOAD, "queries_per_step": n, "grid": list(dense.shape),
                   "grid_storage": "dense float4 {phi,n} FP32, 16 MB",
                   "points": "surface + N(0,(2h)^2) offsets, seed 1, FP32, HBM-resident",
                   "l2": "flushed (256 MB write) before every timed step",
                   "parallelism": f"replicas x{world}"},
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
                     "frac": achieved / peak, "traffic": traffic, "peak_source": peak_src,
                     "kernel": head_kernel,
                     "bytes_per_query": BYTES_PER_QUERY,
                     "note": "16 MB grid is L2-resident after the first touch; achieved "
                             "counts gather-model bytes, DRAM traffic is lower"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": 12 * n,
                "d2h_bytes_per_step": 17 * n, "by_host_io_mode": e2e_modes,
                "path": "sdfo_query_host, pinned host buffers, synchronous; default host io: the "
                        "query kernel reads the points from and writes the results to the pinned "
                        "buffers (mapped into the device) while it runs, both bus directions at once"},
        "gpu_launches": args.steps,
        "step_us": {"min": 1e3 * min(head_steps), "median": 1e3 * float(np.median(head_steps)),
                    "max": 1e3 * max(head_steps)},
        "clocks": clk,
        "build": {
            "dense_voxels_per_s": n_vox / t_dense,
            "dense_ms": 1e3 * t_dense, "dense_setup_alloc_ms": st_dense["setup_ms"],
            "dense_fill_kernel_ms": st_dense["fill_ms"],
            "dense_bvh_ms": st_dense["bvh_ms"], "dense_hessian_ms": st_dense["hessian_ms"],
            "dense_fill_voxels_per_s": n_vox / (1e-3 * st_dense["fill_ms"]),
            "lbvh_dense_ms": 1e3 * t_lbvh, "lbvh_bvh_ms": st_lbvh["bvh_ms"],
            "lbvh_fill_ms": st_lbvh["fill_ms"],
            "sparse_ms": 1e3 * t_sparse, "sparse_blocks": sparse.block_count,
            "sparse_stored_voxels_per_s": sparse.stored_voxels / t_sparse,
            "sparse_fill_ms": st_sparse["fill_ms"],
            "cpu_reference_dense_voxels_per_s": cpu_build,
            "dense_fill_traversal": trav,
            "knobs_fill_ms": knobs,
        },
        "queries": {
            "dense_tricubic_fwd_per_s": n / per_launch_s,
            "sparse_tricubic_fwd_per_s": n / (sparse_ms * 1e-3),
            "ad_fwd_bwd_per_s": n / (ad_ms * 1e-3),
            "ad_fwd_bwd_regather_per_s": n / (ad_rg_ms * 1e-3),
            "fused_jacobian_per_s": n / (jac_ms * 1e-3),
            "fd_jacobian_per_s": n / (fd_ms * 1e-3),
            "ad_vs_fd_speedup": fd_ms / ad_ms,
            "fused_jacobian_vs_fd_speedup": fd_ms / jac_ms,
        },
        "contact": {
            "poses": 4096, "quadrature_points": int(len(cc["quad_x"])),
            "trilinear_fwd_jac_poses_per_s": 4096 / (ct_ad * 1e-3),
            "trilinear_fwd_poses_per_s": 4096 / (ct_fwd * 1e-3),
            "trilinear_fd_jacobian_poses_per_s": 4096 / (ct_fd * 1e-3),
            "ad_vs_fd_speedup": ct_fd / ct_ad,
            "tricubic_fwd_jac_poses_per_s": 4096 / (ct_ad3 * 1e-3),
        },
        "contact_aware": ca,
        "sdfo_io": sdfo_io,
        "be_step": be_out,
        "c4": c4,
        "c5": c5,
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    del sdfo


def kernels_once(which):
    """Setup of a workload, then ONE launch of each query kernel (forward,
    FP16 forward where sparse, linearising forward, saved backward, the
    regathering backward) with a 64 MB buffer written before each -- the
    program an ncu capture (-k regex:"k_query|k_backward") runs.  "ca": one
    contact-aware build of the cylinder (its fill kernels) and one
    ContactAware query launch.  "be": 296 ring drops (two per SM), eight
    BE step launches (the last ones in contact).  "build": one dense and one
    sparse (band 3) reference-order build of the hollow cylinder
    (k_dense_fill, k_dense_hessian, k_sparse_activate, k_sparse_fill);
    "build5": the same sparse build of the 1.31M-triangle icosphere at 512³.
    "c4": the first 16 gears of the 256-gear set, one batched query launch
    (16 x 65,536 points, identity poses).
    "contact": the ring-on-cube contact batch (4096 poses x 7680 points),
    one Trilinear forward, one Trilinear forward + Jacobian and one
    Tricubic forward + Jacobian launch."""
    import ctypes

    import torch

    from sdfo import SdfGrid
    from sdfo import _native as N
    from sdfo import workloads as W

    lib = N.load()
    if which == "c4":
        # the first 16 gears of the 256-gear set, one batched build and ONE
        # posed Tricubic batch launch over 16 x 65,536 near-surface points
        from sdfo.batch import QueryBatch, pack_poses

        gears = W.c4_gears()[:16]
        grids = SdfGrid.build_sparse_batched(
            [dict(verts=g["verts"], tris=g["tris"], **g["sparse"]) for g in gears], mode=TRICUBIC)
        rng = np.random.default_rng(3)
        pts = []
        for g, grid in zip(gears, grids):
            pts.append(W.near_surface_points(g["verts"], g["tris"], float(grid.voxel[0]), 65_536,
                                             int(rng.integers(1 << 30))))
        x = torch.tensor(np.concatenate(pts).astype(np.float32), device="cuda")
        poses = pack_poses(np.array([np.eye(3)] * len(grids)), np.zeros((len(grids), 3)), device="cuda")
        qb = QueryBatch(grids, [65_536] * len(grids))
        out = qb.outputs(x.device)
        torch.empty(64 << 20, dtype=torch.uint8, device="cuda").zero_()
        qb.run(x, poses, TRICUBIC, out)
        torch.cuda.synchronize()
        print(json.dumps({"kernels_once": which, "grids": len(grids), "queries": int(x.shape[0]),
                          "pool_mb": round(16 * sum(g.stored_voxels for g in grids) / 2**20, 1)}))
        return
    if which == "contact":
        from sdfo.contact import ContactBatch, pack_states

        cc = W.c3_ring_cube(n_poses=4096)
        cube = SdfGrid.build_dense(*cc["cube"], **cc["build"])
        poses = pack_states(cc["r"], cc["R"], cc["v"], cc["w"], device="cuda")
        body_b = pack_states(np.zeros((1, 3)), np.eye(3)[None], device="cuda")[0]
        b2 = ContactBatch(cube, cc["quad_x"], cc["quad_w"], mode=2, **cc["params"])
        b3 = ContactBatch(cube, cc["quad_x"], cc["quad_w"], mode=3, **cc["params"])
        b2.evaluate(poses, body_b)
        b2.evaluate(poses, body_b, jacobian=True)
        b3.evaluate(poses, body_b, jacobian=True)
        torch.cuda.synchronize()
        print(json.dumps({"kernels_once": which, "poses": 4096, "points": int(len(cc["quad_x"]))}))
        return
    if which == "build5":
        c = W.c5_icosphere()
        N.check(lib.sdfo_set_bvh_mode(N.BVH_REFERENCE))
        s = SdfGrid.build_sparse(c["verts"], c["tris"], **c["sparse"])
        torch.cuda.synchronize()
        print(json.dumps({"kernels_once": which, "sparse_blocks": s.block_count,
                          "stats": s.build_stats()}))
        return
    if which == "build":
        c = W.c2_cylinder()
        N.check(lib.sdfo_set_bvh_mode(N.BVH_REFERENCE))
        d = SdfGrid.build_dense(c["verts"], c["tris"], **c["dense"])
        s = SdfGrid.build_sparse(c["verts"], c["tris"], **c["sparse"])
        torch.cuda.synchronize()
        print(json.dumps({"kernels_once": which, "dense_voxels": int(np.prod(d.shape)),
                          "sparse_blocks": s.block_count}))
        return
    if which == "be":
        from sdfo.be import BEStepper

        c = W.be_ring_drops(296)
        grid = SdfGrid.build_dense(*c["slab"], **c["build"])
        p = c["params"]
        st = BEStepper(grid, c["quad_x"], c["quad_w"], c["mass"], c["inertia"], p["stiffness"],
                       order=p["order"], damping=p["damping"], friction=p["friction"],
                       regularizer=p["regularizer"], activation_distance=p["activation_distance"],
                       narrow_margin=0.01, max_scenes=296)
        scenes = st.scenes(c["r"], c["R"], c["v"], c["w"])
        for _ in range(8):
            st.step(scenes, 1e-3)
        torch.cuda.synchronize()
        print(json.dumps({"kernels_once": which, "scenes": 296, "steps": 8}))
        return
    if which == "ca":
        from sdfo import meshes as M

        c = W.c2_cylinder()
        cn = M.corner_normals(c["verts"], c["tris"], "face")
        g = SdfGrid.build_contact_aware(c["verts"], c["tris"], cn, **c["dense"])
        pts = torch.tensor(points_for(c, float(g.voxel[0])), device="cuda")
        n = pts.shape[0]
        out = torch.empty(n, device="cuda")
        valid = torch.empty(n, dtype=torch.uint8, device="cuda")
        torch.empty(16 << 20, device="cuda").zero_()
        N.check(lib.sdfo_query(g.handle, 4, ctypes.c_void_p(pts.data_ptr()), 0, n,
                               ctypes.c_void_p(out.data_ptr()), None, None, None,
                               ctypes.c_void_p(valid.data_ptr()), None,
                               ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)))
        torch.cuda.synchronize()
        print(json.dumps({"kernels_once": which, "queries": n}))
        return
    if which == "c2":
        c = W.c2_cylinder()
        grids = [SdfGrid.build_dense(c["verts"], c["tris"], mode=TRICUBIC, **c["dense"])]
        pts = torch.tensor(points_for(c, float(grids[0].voxel[0])), device="cuda")
    else:
        c = W.c5_icosphere()
        g = SdfGrid.build_sparse(c["verts"], c["tris"], mode=TRICUBIC, **c["sparse"])
        grids = [g, g.to_fp16()]
        pts = torch.tensor(W.c5_points(c["verts"], c["tris"], float(g.voxel[0]), n=4_000_000),
                           device="cuda")
    n = pts.shape[0]

    def P(t):
        return ctypes.c_void_p(t.data_ptr())

    s = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    f32 = dict(device="cuda", dtype=torch.float32)
    gap, grad, h6 = torch.empty(n, **f32), torch.empty((n, 3), **f32), torch.empty((n, 6), **f32)
    valid = torch.empty(n, dtype=torch.uint8, device="cuda")
    dgap, dgrad, dp = torch.randn(n, **f32), torch.randn((n, 3), **f32), torch.empty((n, 3), **f32)
    dgrid = torch.zeros((grids[0].stored_voxels, 4), **f32)
    buf = torch.empty(16 << 20, **f32)
    g = grids[0]
    for gg in grids:
        buf.zero_()
        N.check(lib.sdfo_query(gg.handle, TRICUBIC, P(pts), 0, n, P(gap), P(grad), None, None,
                               P(valid), None, s))
    buf.zero_()
    N.check(lib.sdfo_query_linearize(g.handle, TRICUBIC, P(pts), n, P(gap), P(grad), P(valid),
                                     P(h6), s))
    buf.zero_()
    N.check(lib.sdfo_query_backward_saved(g.handle, TRICUBIC, P(pts), n, P(grad), P(h6), P(valid),
                                          P(dgap), P(dgrad), P(dp),
                                          P(dgrid) if which == "c5" else None, s))
    buf.zero_()
    N.check(lib.sdfo_query_backward(g.handle, TRICUBIC, P(pts), n, P(dgap), P(dgrad), P(dp), None,
                                    s))
    torch.cuda.synchronize()
    print(json.dumps({"kernels_once": which, "queries": n}))


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.kernels_once:
        kernels_once(args.kernels_once)
        return
    import torch

    if world > 1:
        torch.cuda.set_device(local_rank)
        torch.distributed.init_process_group("nccl", timeout=datetime.timedelta(seconds=600),
                                             device_id=torch.device("cuda", local_rank))
    try:
        run_ours(args, rank, world, local_rank)
    finally:
        if world > 1:
            torch.distributed.barrier()
            torch.distributed.destroy_process_group()


if __name__ == "__main__":
    main()

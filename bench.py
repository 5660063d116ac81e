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
    ap.add_argument("--steps", type=int, default=200)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
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
def timed(torch, fn, steps, warmup, flush, stream):
    """Sum of per-step CUDA-event durations, L2 flushed before each step."""
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
    return sum(s.elapsed_time(e) for s, e in evs)


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
    total_ms = timed(torch, lambda: query(dense), args.steps, args.warmup, flush, stream)
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

    def ad_step():
        query(dense)
        N.check(lib.sdfo_query_backward(dense.handle, TRICUBIC, P(pts), n, P(dgap), P(dgrad),
                                        P(dpts), None, sptr()))

    ad_ms = timed(torch, ad_step, args.steps, args.warmup, flush, stream) / args.steps
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

    peak, peak_src = measured_peaks()
    achieved = BYTES_PER_QUERY * n / per_launch_s / 1e9
    traffic = ncu_traffic("tricubic_dense_c2")
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
                     "kernel": "k_query<Tricubic,dense>",
                     "bytes_per_query": BYTES_PER_QUERY,
                     "note": "16 MB grid is L2-resident after the first touch; achieved "
                             "counts gather-model bytes, DRAM traffic is lower"},
        "cpu_baseline": cpu,
        "e2e": {"value": e2e_value, "unit": "queries/s", "h2d_bytes_per_step": 12 * n,
                "d2h_bytes_per_step": 17 * n,
                "path": "sdfo_query_host, pinned host buffers, synchronous"},
        "gpu_launches": args.steps,
        "clocks": clk,
        "build": {
            "dense_voxels_per_s": n_vox / t_dense,
            "dense_ms": 1e3 * t_dense, "dense_fill_kernel_ms": st_dense["fill_ms"],
            "dense_bvh_ms": st_dense["bvh_ms"], "dense_hessian_ms": st_dense["hessian_ms"],
            "dense_fill_voxels_per_s": n_vox / (1e-3 * st_dense["fill_ms"]),
            "lbvh_dense_ms": 1e3 * t_lbvh, "lbvh_bvh_ms": st_lbvh["bvh_ms"],
            "lbvh_fill_ms": st_lbvh["fill_ms"],
            "sparse_ms": 1e3 * t_sparse, "sparse_blocks": sparse.block_count,
            "sparse_stored_voxels_per_s": sparse.stored_voxels / t_sparse,
            "sparse_fill_ms": st_sparse["fill_ms"],
            "cpu_reference_dense_voxels_per_s": cpu_build,
        },
        "queries": {
            "dense_tricubic_fwd_per_s": n / per_launch_s,
            "sparse_tricubic_fwd_per_s": n / (sparse_ms * 1e-3),
            "ad_fwd_bwd_per_s": n / (ad_ms * 1e-3),
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
    }
    if rank == 0:
        print(json.dumps(line), flush=True)
    del sdfo


def main():
    args = parse()
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local_rank = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
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

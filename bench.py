"""Benchmark: q.triangle evals/s of the numeric (mesh) form factor on one B200.

Workload (large numeric form factor, DWBA): a seeded closed star-shaped mesh of 50,000
triangles (UV sphere 250 x 101 bands, radius 15 nm perturbed by real spherical harmonics
l <= 8) on a 2048 x 2048 detector (qy in [-2, 2], qz in [0, 3] 1/nm, 10 keV, alpha_i =
0.20 deg, vacuum particle layer), four DWBA qz blocks: 4 * 2048^2 * 50,000 = 8.39e11
q.triangle evaluations per step.  A step is one FP32-compensated triangle sum over the
whole grid, inputs resident in HBM (the q-grid is 332 MB, larger than L2).

Reported beside it: the plain FP64 kernel on the same inputs, the end-to-end number through
the reference-shaped C-ABI call with host buffers (H2D + D2H inside the timed region), the
roofline of the dominant kernel against FP32 and SFU throughput measured on the same GPU,
and the reference's own CPU implementation timed on the host cores on a bounded sample.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl hgx|reference]
Under torchrun (N > 1) every rank runs an independent replica (the form factor needs no
exchange): weak scaling, time = max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NCOL = NROW = 2048
QMIN_Y, QMIN_Z, QMAX_Y, QMAX_Z = -2.0, 0.0, 2.0, 3.0
ENERGY_KEV, ALPHA_I_DEG = 10.0, 0.20
PI_REF = 3.141592653589793
# FP32 FLOP of the row-factorised kernel per (pixel, triangle) for the 4 paired real
# DWBA blocks (FMA = 2): in-plane phase offset q_par.d 3, in-plane q_par.n~ 3, U = (q.n~) E 2,
# 16 FFMA accumulations 32 -> 40 FLOP and 2 SFU ops (sin, cos) per 4 evaluations.  Not
# counted: the explicit reduction on wide tiles, the per-tile anchor rotation and TwoSum fold.
FLOP_PER_PIXEL_TRI = 40.0
SFU_PER_PIXEL_TRI = 2.0
# DRAM bytes per launch of the row kernel: ncu dram__bytes_read.sum + dram__bytes_write.sum
# of one 2048 x 2048 launch with 50,000 triangles (75.2 MB read + 84.8 MB written)
TRAFFIC_BYTES_PER_LAUNCH = 160.0e6
TRAFFIC_SOURCE = "ncu capture of a 2048x2048 launch (75.2 MB read + 84.8 MB write)"
# the library's kernels per form-factor step (bounding box 2, Morton keys, tiles, row kernel);
# CUB's radix sort of the keys adds 6 launches per step
HGX_LAUNCHES_PER_STEP = 5
CUB_LAUNCHES_PER_STEP = 6


# Executed FLOP per unit of the other timed kernels, from ncu thread-instruction counts
# (2 x FMA + MUL + ADD of each precision) of one launch on the bench's own descriptions,
# each from an ncu capture of its kernel on the workload below:
#   mesh_backward_kernel     82.5 FP32 per (pixel, triangle)   (the expression: 80)
#   ff_exact_kernel          611 FP64 per (q-point, triangle)
#   grain_dwba_kernel        6418 FP64 per (pixel, grain), hcp cylinders (HIG_ENSEMBLE)
#   grain_dwba_f32c_kernel   1060 FP32 + 408 FP64 per (pixel, grain), the same description
#   cyl_pixels_f32c_kernel   221 FP32 + 60 FP64 per ROI pixel (the 256-candidate batch)
#   cyl_pixels_kernel<double>  1418 FP64 per ROI pixel (the same batch)
#   grain_dwba_f32c_kernel   1340 FP32 + 554 FP64 and 159 XU-pipe operations per pixel (config 1)
#   grain_dwba_kernel        16999 FP64 per pixel (config 1)
CYL_F32C_FP32_FLOP_PER_PIXEL = 221.0
CYL_F32C_FP64_FLOP_PER_PIXEL = 60.0
CYL_F64_FLOP_PER_PIXEL = 1418.0
CFG1_F32C_FP32_FLOP_PER_PIXEL = 1340.0
CFG1_F32C_FP64_FLOP_PER_PIXEL = 554.0
CFG1_F32C_XU_PER_PIXEL = 159.0
CFG1_F64_FLOP_PER_PIXEL = 16999.0
MESH_FWD_FLOP_PER_PIXEL_TRI = FLOP_PER_PIXEL_TRI
MESH_BWD_FLOP_PER_PIXEL_TRI = 80.0
EXACT_FP64_FLOP_PER_EVAL = 611.0
GRAIN_FP64_FLOP_PER_PIXEL_GRAIN = 6418.0
GRAIN_F32C_FP32_FLOP_PER_PIXEL_GRAIN = 1060.0
GRAIN_F32C_FP64_FLOP_PER_PIXEL_GRAIN = 408.0


def roofline_of(bound, flop_per_unit, units, seconds, peak, unit, source):
    """A roofline sub-object: achieved TFLOP/s = flop_per_unit x units / seconds, its fraction
    of the measured peak of the bounding pipe (the library's own probes on this GPU)."""
    ach = flop_per_unit * units / seconds / 1e12
    return {"bound": bound, "flop_per_unit": flop_per_unit, "unit": unit, "units": units,
            "achieved": ach, "peak": peak, "units_rate": "TFLOP/s", "frac": ach / peak,
            "flop_source": source}


def hbm_view(ms_step):
    """The row kernel against HBM bandwidth (MEASURED_PEAKS.json): its algorithmic bytes per
    launch are the q-grid read once (qx, qy FP64) and the complex64 output written once; the
    measured DRAM traffic is TRAFFIC_BYTES_PER_LAUNCH.  Far below 1: not memory-bound."""
    n = NCOL * NROW
    alg = 2 * 8 * n + 4 * 8 * n
    peak = None
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            peak = float(json.load(f)["hbm_gbs"])
    except (OSError, KeyError, ValueError):
        pass
    achieved = alg / (ms_step * 1e-3) / 1e9
    return {"bound": "hbm", "algorithmic_bytes": alg, "achieved": achieved, "unit": "GB/s",
            "peak": peak, "frac": None if peak is None else achieved / peak,
            "peak_source": "MEASURED_PEAKS.json hbm_gbs (measured copy)"}


def max_over_ranks(x, dist, device):
    """The largest x over all ranks (the slowest replica's time); x itself without a process
    group.  Every rank must call it at the same point."""
    if dist is None:
        return float(x)
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def job_throughput(world, units_per_rank, seconds_max):
    """Whole-job rate of independent replicas: all ranks' units over the slowest rank's time."""
    return world * units_per_rank / seconds_max


def k0_from_kev(e):
    return 2 * PI_REF / (1.23984 / e)


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="hgx", choices=["hgx", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-f64", action="store_true")
    ap.add_argument("--no-fitting", action="store_true")
    ap.add_argument("--no-exact", action="store_true")
    ap.add_argument("--no-hig", action="store_true")
    ap.add_argument("--no-config1", action="store_true")
    ap.add_argument("--grid", type=int, default=0,
                    help="detector rows = columns of the form-factor workload (default 2048; "
                         "smaller grids are for profiling captures, not bench lines)")
    ap.add_argument("--ppt", type=int, default=0,
                    help="row-kernel pixels per thread (0: the library's autotuner chooses)")
    return ap.parse_args()


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = index
        self.proc = None
        self.path = None

    def start(self):
        try:
            fd, self.path = tempfile.mkstemp(suffix=".csv")
            os.close(fd)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f,
                stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None

    def stop(self):
        if self.proc is None:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        self.f.close()
        rows = []
        for line in open(self.path):
            p = [x.strip() for x in line.split(",")]
            if len(p) >= 9:
                rows.append(p)
        os.unlink(self.path)
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in rows if r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i] == "Active"})
        load = [s for s in sm]
        return {"sm_mhz": float(np.median(load)) if load else None,
                "sm_max_mhz": max(mx) if mx else None, "reasons": reasons,
                "samples": len(rows)}


def workload_mesh():
    from hipgisaxs_b200 import meshes
    V, F = meshes.star_mesh(15.0, 250, 101, 8, 0.05, meshes.DEFAULT_SEED)
    return meshes.shape_def_from_mesh(V, F)


def cpu_sample_rate(sd, qx, qy, qz_ext, budget_s=12.0, backend=None):
    """Times the reference's compute_approx_triangle (oracle/_ref, else the port) on whole
    detector rows of the workload; returns (evals/s, threads, kind, sample description)."""
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    kind = "reference" if po.available("ref") else "port"
    be = "ref" if kind == "reference" else "port"
    threads = po.set_threads(os.cpu_count() or 1, be)
    n = NCOL * NROW
    ext = qz_ext.reshape(4, n)

    def run(rows):
        idx = np.concatenate([np.arange(r * NCOL, (r + 1) * NCOL) for r in rows])
        qz = ext[:, idx].ravel()
        t = time.perf_counter()
        po.ff_approx_triangle(sd, qx[idx], qy[idx], qz, None, be)
        dt = time.perf_counter() - t
        return 4 * len(idx) * len(sd), dt

    ev, dt = run([NROW // 2])
    nrows = int(max(1, min(64, budget_s / max(dt, 1e-3))))
    rows = list(np.linspace(0, NROW - 1, nrows).astype(int))
    ev, dt = run(rows)
    desc = (f"{nrows} full detector rows x 4 DWBA blocks x {len(sd)} triangles "
            f"({ev:.3e} evals, {dt:.1f} s); cost is linear in q-points")
    return ev / dt, threads, kind, desc


def fitting_bench(ctx, torch, dev, stream, steps=5):
    """Configs 3 and 4: chi^2 + gradient of the cylinder-lattice model (R 5, H 10 nm, 5% size
    spread over 11 samples, hex lattice a = 20 nm, 20 x 20 repetitions, Si-like substrate,
    10 keV, alpha_i 0.20 deg, 1024 x 1024 detector) against a Poisson target (peak 1e4 counts)
    simulated at R*1.03, H*0.96, a*1.02, phi + 5 deg.  The fused FP32C forward + adjoint is
    timed against the plain FP64 form with the reference fitter's central differences
    (1 + 2*4 forward runs + chi^2 each)."""
    import hipgisaxs_b200 as hg
    from hipgisaxs_b200 import fitting, model
    n = 1024
    alpha_i = ALPHA_I_DEG * PI_REF / 180
    k0 = k0_from_kev(ENERGY_KEV)
    g = hg.QGrid.create(ctx, n, n, QMIN_Y, QMIN_Z, QMAX_Y, QMAX_Z, alpha_i, k0)
    rowfc = model.propagation_coeffs(ctx, g, [(4.88e-6, 7.37e-8, 0.0, -1)], k0, alpha_i, 0,
                                     per_row=True)
    abc, _ = model.lattice_vectors("hex")
    dn2 = (-2 * 4.88e-6, -2 * 7.37e-8)

    def mb(R, H, a, phi):
        # 11 evenly spaced size samples (smooth in R and H; see include/hgx.h model slot 15)
        return fitting.model_block(R, H, a, phi, 0.05, 11, (20, 20, 1), dn2, (0, 0, 0), 1.0,
                                   smooth_sampling=True)

    p0 = mb(5.0, 10.0, 20.0, 0.0)
    truth = mb(5.0 * 1.03, 10.0 * 0.96, 20.0 * 1.02, np.deg2rad(5.0))
    full = [0, 0, n, n]
    fwd = fitting.CylinderBatch(ctx, g, rowfc, abc, [full], precision="f64")
    target = fwd.forward([truth])[0].ravel()
    rng = np.random.default_rng(20240601)
    scale = 1e4 / target.max()
    counts = rng.poisson(scale * target).astype(np.float64)
    fwd.close()

    out = {}
    # ---- config 3: one candidate, full detector
    b32 = fitting.CylinderBatch(ctx, g, rowfc, abc, [full], counts, None, scale, "f32c")
    b64 = fitting.CylinderBatch(ctx, g, rowfc, abc, [full], counts, None, scale, "f64")
    b32.tune([p0], reps=2)
    c32, g32 = b32.eval([p0])
    c64, g64 = b64.eval([p0])

    def timed(fn, n):
        for _ in range(3):
            fn()
        t = time.perf_counter()
        for _ in range(n):
            fn()
        return (time.perf_counter() - t) / n

    dt32 = timed(lambda: b32.eval([p0]), steps)
    dt64 = timed(lambda: b64.eval([p0]), steps)  # the same fused forward + adjoint in FP64
    # plain FP64 form, central differences: 9 forwards + chi^2 on the device
    d_counts = torch.tensor(counts, device=dev)
    d_I = torch.empty(n * n, dtype=torch.float64, device=dev)

    def chi2_plain(m):
        hg._capi.check(hg.lib().hgx_cyl_plain_forward(b64._h, 0, np.ascontiguousarray(m).ctypes.data,
                                                      d_I.data_ptr()))
        return model.chi2(ctx, d_I, d_counts, None, scale)

    def fd_grad(m):
        c = chi2_plain(m)
        gr = np.zeros(4)
        for j in range(4):
            h = 1e-4 * (abs(m[j]) if j < 3 else 1.0)
            mp, mm = m.copy(), m.copy()
            mp[j] += h
            mm[j] -= h
            gr[j] = (chi2_plain(mp) - chi2_plain(mm)) / (2 * h)
        return c, gr

    fd_grad(p0)
    t = time.perf_counter()
    cfd, gfd = fd_grad(p0)
    dtfd = time.perf_counter() - t
    out["chi2_grad_1024sq"] = {
        "metric": "chi2+grad evals/s", "value": 1.0 / dt32, "ms_per_eval": 1e3 * dt32,
        "plain_fp64_fd": {"value": 1.0 / dtfd, "ms_per_eval": 1e3 * dtfd,
                          "method": "plain FP64 forward x 9 (central differences, h 1e-4 rel)"},
        "speedup_vs_plain_fp64": dtfd / dt32,
        "fp64_adjoint": {"value": 1.0 / dt64, "ms_per_eval": 1e3 * dt64,
                         "method": "the same fused forward + adjoint in FP64: every Bessel function "
                                   "and Dirichlet kernel per pixel (no radial tables)"},
        "speedup_vs_fp64_adjoint": dt64 / dt32,
        "rel_err_chi2_vs_fp64": abs(c32[0] - c64[0]) / abs(c64[0]),
        "rel_err_grad_vs_fp64": float(np.linalg.norm(g32 - g64) / np.linalg.norm(g64)),
        "fd_vs_adjoint_rel": float(np.linalg.norm(gfd - g64[0]) / np.linalg.norm(g64[0])),
        "pixels": n * n, "params": 4}
    b32.close()
    b64.close()

    # ---- config 4: 256 candidates with uneven ROIs in one graph-captured launch
    rng = np.random.default_rng(20240602)
    nc = 256
    ny = rng.integers(128, 1025, nc)
    nz = rng.integers(128, 1025, nc)
    rois = np.array([[rng.integers(0, n - z + 1), rng.integers(0, n - y + 1), z, y]
                     for y, z in zip(ny, nz)], dtype=np.int32)
    cimg = counts.reshape(n, n)
    cat = np.concatenate([cimg[r0:r0 + z, c0:c0 + y].ravel() for r0, c0, z, y in rois])
    f = 1 + rng.uniform(-0.1, 0.1, (nc, 3))
    models = np.array([mb(5.0 * f[i, 0], 10.0 * f[i, 1], 20.0 * f[i, 2],
                          np.deg2rad(rng.uniform(-10, 10))) for i in range(nc)])
    bb32 = fitting.CylinderBatch(ctx, g, rowfc, abc, rois, cat, None, scale, "f32c")
    bb64 = fitting.CylinderBatch(ctx, g, rowfc, abc, rois, cat, None, scale, "f64")
    # tile shape of the persistent pixel pass chosen by the library's autotuner on this batch
    shapes = fitting.CylinderBatch.shapes()
    tbest, _, ttimes = bb32.tune(models, reps=2)
    cc32, gg32 = bb32.eval(models)
    cc64, gg64 = bb64.eval(models)
    dtb = timed(lambda: bb32.eval(models), steps)
    dtb64 = timed(lambda: bb64.eval(models), steps)
    # 256 sequential plain launches: the plain FP64 central-difference evaluation of a
    # subsample of candidates, scaled by pixel count
    sub = 8
    pix = rois[:, 2].astype(np.int64) * rois[:, 3]
    # set-up (single-candidate objects, buffers) outside the timed region: the baseline is
    # the plain FP64 forward and chi^2, nine times per candidate
    plain = []
    for i in range(sub):
        r0, c0, z, y = rois[i]
        cb = fitting.CylinderBatch(ctx, g, rowfc, abc, [rois[i]],
                                   cat[bb32.offsets[i]:bb32.offsets[i + 1]], None, scale, "f64")
        dI = torch.empty(int(z) * int(y), dtype=torch.float64, device=dev)
        dC = torch.tensor(cat[bb32.offsets[i]:bb32.offsets[i + 1]], device=dev)
        plain.append((cb, dI, dC))
    torch.cuda.synchronize()
    t = time.perf_counter()
    for i, (cb, dI, dC) in enumerate(plain):
        for j in range(9):
            m = models[i].copy()
            if j:
                k = (j - 1) // 2
                m[k] += (1 if j % 2 else -1) * 1e-4 * (abs(m[k]) if k < 3 else 1.0)
            hg._capi.check(hg.lib().hgx_cyl_plain_forward(cb._h, 0, np.ascontiguousarray(m).ctypes.data,
                                                          dI.data_ptr()))
            model.chi2(ctx, dI, dC, None, scale)
    dts = (time.perf_counter() - t) * pix.sum() / pix[:sub].sum()
    for cb, _, _ in plain:
        cb.close()
    rel_c = float(np.max(np.abs(cc32 - cc64) / np.abs(cc64)))
    rel_g = float(np.max(np.linalg.norm(gg32 - gg64, axis=1) / np.linalg.norm(gg64, axis=1)))
    out["batch_256_rois"] = {
        "metric": "chi2+grad evals/s", "value": nc / dtb, "ms_per_batch": 1e3 * dtb,
        "candidates": nc, "pixels": int(pix.sum()), "work_items": bb32.nitems,
        "tile_shape": {"threads": shapes[tbest][0], "pixels_per_thread": shapes[tbest][1],
                       "autotuner_ms": {f"{t}x{p}": v for (t, p), v in zip(shapes, ttimes)}},
        "sequential_plain_fp64_fd": {"value": nc / dts, "s_per_batch": dts,
                                     "sample": f"{sub} candidates timed, scaled by pixels"},
        "speedup_vs_sequential_plain": dts / dtb,
        "fp64_adjoint": {"value": nc / dtb64, "ms_per_batch": 1e3 * dtb64,
                         "method": "the same graph-captured batch in FP64: every Bessel function and "
                                            "Dirichlet kernel per pixel (no radial tables)"},
        "speedup_vs_fp64_adjoint": dtb64 / dtb,
        "max_rel_err_chi2_vs_fp64": rel_c, "max_rel_err_grad_vs_fp64": rel_g}
    bb32.close()
    bb64.close()
    g.close()
    return out


def exact_bench(ctx, torch, stream, sd_mesh, steps=2, n=512):
    """The exact (polyhedral) triangle form factor, FP64: the 50,000-triangle star mesh on an
    n x n DWBA detector of the headline's q-range (4 n^2 x 50,000 evaluations), device-resident
    inputs, CUDA events; beside it the reference's own compute_exact_triangle (oracle/_ref,
    all host threads) on whole detector rows of the same workload."""
    import hipgisaxs_b200 as hg
    from hipgisaxs_b200 import meshes
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    V, F = meshes.star_mesh(15.0, 250, 101, 8, 0.05, meshes.DEFAULT_SEED)
    tris = po.mesh_triangles(V, F)
    alpha_i = ALPHA_I_DEG * PI_REF / 180
    g = hg.QGrid.create(ctx, n, n, QMIN_Y, QMIN_Z, QMAX_Y, QMAX_Z, alpha_i, k0_from_kev(ENERGY_KEV))
    dev = torch.device("cuda", torch.cuda.current_device())
    d_tris = torch.tensor(tris, device=dev)
    out = torch.empty(4 * n * n, dtype=torch.complex128, device=dev)
    hg.ff_exact_triangles(ctx, g, d_tris, None, out=out)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(steps):
        hg.ff_exact_triangles(ctx, g, d_tris, None, out=out)
    e1.record(stream)
    torch.cuda.synchronize()
    ms = e0.elapsed_time(e1) / steps
    evals = 4.0 * n * n * len(tris)
    res = {"metric": "q.triangle evals/s", "value": evals / (ms * 1e-3), "ms_per_step": ms,
           "dtype": "f64", "workload": f"star mesh {len(tris)} triangles, {n}x{n} DWBA grid"}
    if po.available("ref"):
        r = g.read(qz_det=False, alpha=False)
        ext = r["qz_ext"].reshape(4, n * n)
        threads = po.set_threads(os.cpu_count() or 1, "ref")
        rows = [n // 3, (2 * n) // 3]
        idx = np.concatenate([np.arange(x * n, (x + 1) * n) for x in rows])
        t = time.perf_counter()
        po.ff_exact_triangle(tris, r["qx"][idx], r["qy"][idx], ext[:, idx].ravel(), None, "ref")
        dt = time.perf_counter() - t
        cev = 4.0 * len(idx) * len(tris)
        res["cpu_reference"] = {"value": cev / dt, "cores": threads,
                                "sample": f"{len(rows)} detector rows x 4 blocks x {len(tris)} "
                                          f"triangles ({cev:.3e} evals, {dt:.1f} s)"}
        res["speedup_vs_cpu_reference"] = res["value"] / res["cpu_reference"]["value"]
    g.close()
    return res


# An ensemble simulation driven by a HiG description of the size of the reference's
# hcp-cylinder example: 600 x 300 detector, 25 x 25 grains with z-rotations drawn over
# [0, 180] degrees, an hcp lattice of 100 x 10 x 2 cells, DWBA over a substrate.
HIG_ENSEMBLE = """hipGisaxsInput = {
	shape = { key = "cyl", name = "cylinder", refindex = { delta = 8.5E-06, beta = 3.1E-07 },
		param = { type = "radius", min = 5 }, param = { type = "height", min = 150 } },
	unitcell = { key = "u1", element = { shape:key = "cyl", locations = [[0 0 0]] } },
	layer = { key = "substr", order = -1, refindex = { delta = 9.1E-06, beta = 2.5E-07 } },
	structure = { key = "st1",
		grain = { unitcell:key = "u1", lattice = { type = "hcp" }, repetition = [100 10 2], scaling = 50 },
		ensemble = { maxgrains = [NG NG 1],
			orientations = { stat = "range", rot1 = { axis = "z", angles = [0 180] } } } },
	instrumentation = { scattering = { alphai = { min = 0.175 }, photon = { value = 7350, unit = "ev" } },
		detector = { pixelsize = 0.172, sdd = 4128.62, directbeam = [ 489.9 843.1 ] } },
	computation = { runname = "ensemble", outputregion = { type = "qspace", minpoint = [ -1 0 ], maxpoint = [ 1 1 ] },
		resolution = [ 600 300 ] }
}
"""


def hig_bench(ctx, steps=3, ng=25):
    """HipGISAXS::compute_gisaxs of HIG_ENSEMBLE through hgx_hig_compute_gisaxs (host image
    out, the call synchronous), timed by the host clock; beside it the oracle's composition
    of the same simulation on one grain (all host threads), scaled to the grain count."""
    import ctypes
    import tempfile
    from hipgisaxs_b200.hig import read_hig
    libc = ctypes.CDLL(None)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "ensemble.hig")
        with open(path, "w") as f:
            f.write(HIG_ENSEMBLE.replace("NG", str(ng)))
        d = read_hig(path)
        nrow, ncol = d.image_size()
        img = np.zeros((nrow, ncol))
        libc.srand(1)
        d.compute_gisaxs(ctx, out=img)
        ts = []
        for _ in range(steps):
            libc.srand(1)
            t = time.perf_counter()
            d.compute_gisaxs(ctx, out=img)
            ts.append(time.perf_counter() - t)
        ms = 1e3 * min(ts)
        grains = ng * ng
        res = {"metric": "simulations/s", "value": 1e3 / ms, "ms_per_simulation": ms,
               "ms_per_grain": ms / grains, "grains": grains, "pixels": nrow * ncol,
               "q_grain_evals_per_s": 4.0 * nrow * ncol * grains / (ms * 1e-3), "dtype": "f64",
               "path": "hgx_hig_compute_gisaxs (fused grain kernel), host image out",
               "workload": f"cylinders on an hcp lattice, {grains} grains, {ncol}x{nrow} DWBA"}
        # the same simulation in FP32C (the fused grain kernel's cylinder and lattice bodies)
        img32 = np.zeros((nrow, ncol))
        libc.srand(1)
        d.compute_gisaxs(ctx, precision="f32c", out=img32)
        ts = []
        for _ in range(steps):
            libc.srand(1)
            t = time.perf_counter()
            d.compute_gisaxs(ctx, precision="f32c", out=img32)
            ts.append(time.perf_counter() - t)
        ms32 = 1e3 * min(ts)
        den = float(np.linalg.norm(img))
        res["f32c"] = {"ms_per_simulation": ms32, "value": 1e3 / ms32,
                       "speedup_vs_f64": ms / ms32,
                       "rel_err_vs_f64": float(np.linalg.norm(img32 - img)) / den,
                       "max_rel_err_vs_f64": float(np.abs(img32 - img).max() / np.abs(img).max())}
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import pyoracle as po
        one = os.path.join(tmp, "one.hig")
        with open(one, "w") as f:
            f.write(HIG_ENSEMBLE.replace("NG", "1"))
        d1 = read_hig(one)
        threads = po.set_threads(os.cpu_count() or 1, "port")
        libc.srand(1)
        t = time.perf_counter()
        po.compute_gisaxs(d1.data, tmp)
        dt = time.perf_counter() - t
        res["cpu_oracle"] = {"s_per_grain": dt, "estimate_s": dt * grains, "cores": threads,
                             "kind": "port",
                             "sample": f"the same description with 1 grain ({dt:.2f} s), x {grains}"}
        res["speedup_vs_cpu_oracle"] = dt * grains / (ms * 1e-3)
    return res


# Config 1: cylinders (R 5 nm, H 10 nm, 5 % Gaussian size spread sampled at 11 values over
# +-3 sigma, summed unweighted as the reference does) on a 2-D hexagonal lattice a = 20 nm with
# 20 x 20 repetitions, one grain, over a Si-like substrate (delta 4.88e-6, beta 7.37e-8, also
# the particles' index), 10 keV, alpha_i 0.20 deg, 1024 x 1024 detector over qy in [-2, 2],
# qz in [0, 3] nm^-1, DWBA.
CONFIG1_HIG = """hipGisaxsInput = {
	shape = { key = "cyl", name = "cylinder", refindex = { delta = 4.88E-06, beta = 7.37E-08 },
		param = { type = "radius", stat = "gaussian", min = 4.25, max = 5.75, p1 = 5, p2 = 0.25, nvalues = 11 },
		param = { type = "height", stat = "gaussian", min = 8.5, max = 11.5, p1 = 10, p2 = 0.5, nvalues = 11 } },
	unitcell = { key = "u1", element = { shape:key = "cyl", locations = [[0 0 0]] } },
	layer = { key = "substr", order = -1, refindex = { delta = 4.88E-06, beta = 7.37E-08 } },
	structure = { key = "st1",
		grain = { unitcell:key = "u1", lattice = { type = "hex" }, repetition = [20 20 1], scaling = 20 },
		ensemble = { maxgrains = [1 1 1] } },
	instrumentation = { scattering = { alphai = { min = 0.2 }, photon = { value = 10000, unit = "ev" } },
		detector = { pixelsize = 0.172, sdd = 4000, directbeam = [ 0 0 ] } },
	computation = { runname = "config1", outputregion = { type = "qspace", minpoint = [ -2 0 ], maxpoint = [ 2 3 ] },
		resolution = [ NRES NRES ] }
}
"""


# The population leg: config 1's description at 512 x 512 with a fitting block over the
# lattice constant (the grain scaling).  (The cylinder's size distribution is summed unweighted,
# as the reference sums it, so moving a Gaussian mean would not change the image.)
POP_FIT = """	fitting = {
		fitparam = { key = "a_lat", variable = "structure['st1']:grain:scaling", range = { min = 19, max = 21 }, init = 20 },
		algorithm = { algoname = "pso", distancemetric = "sqrt_unit_l2" }
	}
}
"""


def population_bench(ctx, npop=64, n=512, steps=3):
    """A PSO generation of npop candidates of config 1's description through
    hgx_hig_population_eval (one recorded graph), FP64 and FP32C, against the reference's way:
    one objective call (one simulation and one distance) per particle (hgx_hig_objective)."""
    import tempfile
    from hipgisaxs_b200.hig import read_hig
    text = CONFIG1_HIG.replace("NRES", str(n)).rstrip().rstrip("}").rstrip() + ",\n" + POP_FIT
    rng = np.random.default_rng(20240605)
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "pop.hig")
        with open(path, "w") as f:
            f.write(text)
        d = read_hig(path)
        d.fit_update([20.3])
        ref = d.compute_gisaxs(ctx).ravel()
        X = rng.uniform(19.2, 20.8, (npop, 1))
        res = {"metric": "objective evals/s", "candidates": npop, "pixels": n * n,
               "workload": f"config 1 description at {n}x{n}, fit parameter: the lattice constant",
               "distance": "sqrt_unit_l2"}
        for prec in ("f64", "f32c"):
            pop = d.population(ctx, npop, ref, None, "sqrt_unit_l2", 0.0, prec)
            v = pop.eval(X)  # records the graph
            best = float("inf")
            for _ in range(steps):
                t = time.perf_counter()
                v = pop.eval(X)
                best = min(best, time.perf_counter() - t)
            pop.close()
            res[prec] = {"ms_per_generation": 1e3 * best, "value": npop / best}
            res[prec + "_dist"] = v
        d.objective(ctx, X[0], ref)
        t = time.perf_counter()
        seq = np.array([d.objective(ctx, x, ref)[0] for x in X])
        dts = time.perf_counter() - t
        res["sequential_objective_calls"] = {"ms_per_generation": 1e3 * dts, "value": npop / dts,
                                             "method": "hgx_hig_objective once per candidate (FP64), "
                                                       "as the reference's PSO loop calls its objective"}
        res["speedup_vs_sequential"] = dts / (res["f64"]["ms_per_generation"] * 1e-3)
        res["fp32c_speedup_vs_fp64"] = res["f64"]["ms_per_generation"] / res["f32c"]["ms_per_generation"]
        d64 = res.pop("f64_dist")
        d32 = res.pop("f32c_dist")
        res["max_rel_diff_vs_sequential"] = float(np.max(np.abs(d64 - seq) / np.abs(seq)))
        res["max_rel_err_fp32c_vs_fp64"] = float(np.max(np.abs(d32 - d64) / np.abs(d64)))
        res["value"] = res["f64"]["value"]
        d.close()
    return res


def config1_bench(ctx, steps=3, n=1024, cpu=True, dev_steps=20):
    """Config 1 through HipGISAXS::compute_gisaxs (hgx_hig_compute_gisaxs, host image out, the
    call synchronous; best of `steps` by the host clock), FP32C and FP64 on the same
    description; beside them the reference's own CPU functions at full size (oracle/_ref:
    AnalyticFormFactor cylinder, StructureFactor, MultiLayer::propagation_coeffs, all host
    threads) with the restated DWBA combination, which is also the accuracy reference."""
    import tempfile
    from hipgisaxs_b200.hig import read_hig
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    res = {"metric": "pixel-evals/s", "workload": "cylinders R 5 H 10 (5% spread, 11 samples), "
           "hex lattice a 20 nm x 20 x 20, Si-like substrate, 10 keV, alpha_i 0.20 deg, "
           f"{n}x{n} DWBA", "pixels": n * n}
    import torch
    stream = torch.cuda.current_stream()
    dimg = torch.empty(n * n, dtype=torch.float64, device="cuda")
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "config1.hig")
        with open(path, "w") as f:
            f.write(CONFIG1_HIG.replace("NRES", str(n)))
        d = read_hig(path)
        imgs = {}
        for prec in ("f32c", "f64"):
            imgs[prec] = d.compute_gisaxs(ctx, precision=prec)
            # device-resident image: CUDA events on the context's stream around the call
            d.compute_gisaxs(ctx, precision=prec, out=dimg)
            torch.cuda.synchronize()
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            for _ in range(dev_steps):
                d.compute_gisaxs(ctx, precision=prec, out=dimg)
            e1.record(stream)
            torch.cuda.synchronize()
            ms_dev = e0.elapsed_time(e1) / dev_steps
            # end to end: the image copied to host memory inside the call
            best = float("inf")
            for _ in range(steps):
                t = time.perf_counter()
                d.compute_gisaxs(ctx, precision=prec)
                best = min(best, time.perf_counter() - t)
            res[prec] = {"ms": ms_dev, "value": n * n / (ms_dev * 1e-3),
                         "e2e_ms_host_image": 1e3 * best}
        d.close()
    i32, i64 = imgs["f32c"].ravel(), imgs["f64"].ravel()
    res["value"] = res["f32c"]["value"]
    res["fp32c_speedup_vs_fp64"] = res["f64"]["ms"] / res["f32c"]["ms"]
    res["fp32c_vs_fp64_note"] = ("beside FP32 arithmetic the FP32C grain kernel sums the cylinder heights in "
                                 "closed form; the FP64 kernel keeps the reference's per-sample height sums "
                                 "(1e-11 parity); both share the in-plane sums across a pixel's four lanes")
    res["timing"] = (f"device image: {dev_steps} back-to-back calls between CUDA events on the launching "
                     "stream (each call returns once queued: tables, grain kernel, structure sum); "
                     "e2e_ms_host_image: one synchronous call with the 8 MB image copied to pageable "
                     "host memory, best of a few, host clock")
    res["rel_err_fp32c_vs_fp64"] = po.rel_err(i32, i64)
    res["max_rel_err_fp32c_vs_fp64"] = float(np.abs(i32 - i64).max() / np.abs(i64).max())
    if cpu and po.available("ref"):
        threads = po.set_threads(os.cpu_count() or 1, "ref")
        G = po.Grid(n, n, -2.0, 0.0, 2.0, 3.0, 0.2, 10.0, backend="ref")
        t = time.perf_counter()
        ff = po.ff_analytic(G, "cylinder", po.cylinder_params(5.0, 10.0, 0.05, 11))
        a, b, c, _ = po.lattice_vectors("hex")
        sf = po.sf_lattice(G, (a, b, c), (20, 20, 1), (20.0, 20.0, 20.0))
        fc = po.propagation_coeffs(G, [(4.88e-6, 7.37e-8, 0.0, -1)], 0)
        ref = po.dwba_combine(fc, sf, complex(-2 * 4.88e-6, -2 * 7.37e-8) * ff, 1.0)
        dt = time.perf_counter() - t
        res["cpu_reference"] = {"value": n * n / dt, "ms": 1e3 * dt, "cores": threads,
                                "kind": "reference", "sample": f"the full {n}x{n} image"}
        res["speedup_vs_cpu_reference"] = res["value"] / res["cpu_reference"]["value"]
        res["rel_err_fp32c_vs_reference"] = po.rel_err(i32, ref)
        res["rel_err_fp64_vs_reference"] = po.rel_err(i64, ref)
    return res


def mesh_grad_bench(ctx, grid, steps=2):
    """Config 3, mesh part: chi^2 and the gradient with respect to all 25,002 x 3 vertex
    coordinates of the 50,000-triangle star mesh on the 2048 x 2048 DWBA detector (forward
    FP32C form factor + adjoint).  The reference's method (central differences) would need
    1 + 2 x 75,006 forward runs; its cost is extrapolated from the forward time."""
    from hipgisaxs_b200 import fitting, meshes, model
    V, F = meshes.star_mesh(15.0, 250, 101, 8, 0.05, meshes.DEFAULT_SEED)
    alpha_i = ALPHA_I_DEG * PI_REF / 180
    k0 = k0_from_kev(ENERGY_KEV)
    rowfc = model.propagation_coeffs(ctx, grid, [(4.88e-6, 7.37e-8, 0.0, -1)], k0, alpha_i, 0,
                                     per_row=True)
    dn2 = (-2 * 4.88e-6, -2 * 7.37e-8)
    Vt, _ = meshes.star_mesh(15.0 * 1.02, 250, 101, 8, 0.05, meshes.DEFAULT_SEED + 1)
    _, _, It = fitting.mesh_chi2_grad(ctx, grid, Vt, F, rowfc, dn2, None, None, 1.0, 1.0,
                                      want_grad=False, want_intensity=True)
    rng = np.random.default_rng(20240603)
    scale = 1e4 / It.max()
    counts = rng.poisson(scale * It).astype(np.float64)
    fitting.mesh_chi2_grad(ctx, grid, V, F, rowfc, dn2, counts, None, scale)
    t = time.perf_counter()
    for _ in range(steps):
        chi, gv, _ = fitting.mesh_chi2_grad(ctx, grid, V, F, rowfc, dn2, counts, None, scale)
    dt = (time.perf_counter() - t) / steps
    dtf = float("inf")
    for _ in range(2):
        t = time.perf_counter()
        fitting.mesh_chi2_grad(ctx, grid, V, F, rowfc, dn2, counts, None, scale, want_grad=False)
        dtf = min(dtf, time.perf_counter() - t)
    # the plain FP64 forward + adjoint once on the same inputs (its own warm-up call first)
    fitting.mesh_chi2_grad(ctx, grid, V, F, rowfc, dn2, counts, None, scale, want_grad=False,
                           precision="f64")
    t = time.perf_counter()
    chi64, gv64, _ = fitting.mesh_chi2_grad(ctx, grid, V, F, rowfc, dn2, counts, None, scale,
                                            precision="f64")
    dt64 = time.perf_counter() - t
    nparam = 3 * len(V)
    return {"metric": "chi2+grad evals/s", "value": 1.0 / dt, "s_per_eval": dt,
            "fp64_adjoint": {"s_per_eval": dt64, "method": "plain FP64 form factor, seeds and "
                             "backward pass on the same inputs (one timed call)"},
            "speedup_vs_fp64_adjoint": dt64 / dt,
            "rel_err_chi2_vs_fp64": abs(chi - chi64) / abs(chi64),
            "rel_err_grad_vs_fp64": float(np.linalg.norm(gv - gv64) / np.linalg.norm(gv64)),
            "forward_only_s": dtf, "vertices": len(V), "triangles": len(F),
            "gradient_components": nparam,
            "central_differences_estimate_s": (1 + 2 * nparam) * dtf,
            "note": "the central-difference gradient was not run: extrapolated from the timed "
                    "forward (1 + 2 x 75,006 forward runs)"}


def run_reference(args, rank):
    """The reference's own CPU implementation of the path on this host's cores."""
    if rank != 0:
        return
    sd = workload_mesh()
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import pyoracle as po
    G = po.Grid(NCOL, NROW, QMIN_Y, QMIN_Z, QMAX_Y, QMAX_Z, ALPHA_I_DEG, ENERGY_KEV)
    kind = "reference" if po.available("ref") else "port"
    be = "ref" if kind == "reference" else "port"
    threads = po.set_threads(os.cpu_count() or 1, be)
    n = NCOL * NROW
    ext = G.qz_ext.reshape(4, n)
    # each step: 2 full detector rows (spread over the detector) x 4 blocks x all triangles
    def step(i):
        r = [(i * 997 + 13) % NROW, (i * 389 + 1024) % NROW]
        idx = np.concatenate([np.arange(x * NCOL, (x + 1) * NCOL) for x in r])
        po.ff_approx_triangle(sd, G.qx[idx], G.qy[idx], ext[:, idx].ravel(), None, be)
        return 4 * len(idx) * len(sd)

    for i in range(args.warmup):
        step(i)
    t = time.perf_counter()
    ev = 0
    for i in range(args.steps):
        ev += step(args.warmup + i)
    dt = time.perf_counter() - t
    v = ev / dt
    sample = "2 full detector rows x 4 DWBA blocks x 50,000 triangles per step"
    line = {"metric": "q.triangle evals/s", "value": v, "unit": "evals/s",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1e3 * dt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "impl": "reference",
            "config": {"workload": "mesh50k-dwba-2048sq (bounded sample per step)",
                       "triangles": len(sd), "grid": [NCOL, NROW], "blocks": 4},
            "cpu_baseline": {"value": v, "unit": "evals/s", "cores": threads, "kind": kind,
                             "sample": sample},
            "e2e": {"value": v, "unit": "evals/s", "h2d_bytes_per_step": 0,
                    "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    global NCOL, NROW
    args = parse()
    if args.grid:
        NCOL = NROW = args.grid
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank)
        return

    import torch
    import hipgisaxs_b200 as hg

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
    dev = torch.device("cuda", local)
    stream = torch.cuda.current_stream(dev)
    ctx = hg.Context(local, stream=stream)

    sd = workload_mesh()
    ntri = len(sd)
    alpha_i = ALPHA_I_DEG * PI_REF / 180
    k0 = k0_from_kev(ENERGY_KEV)
    grid = hg.QGrid.create(ctx, NCOL, NROW, QMIN_Y, QMIN_Z, QMAX_Y, QMAX_Z, alpha_i, k0)
    assert grid.mode == 1, grid.mode
    n = NCOL * NROW
    evals = 4.0 * n * ntri
    sd_dev = torch.tensor(sd, device=dev)
    out = torch.empty(4 * n, dtype=torch.complex64, device=dev)

    # launch shape chosen by the library's autotuner on this grid (outside the timed region;
    # 8,192 triangles rank the candidates, whose cost is linear in the triangle count)
    if args.ppt:
        tuned_p, tune_times = args.ppt, {}
    else:
        tuned_p, _, tune_times = hg.ff_tune(ctx, grid, sd_dev[:8192], None, "c64", reps=2)

    def step():
        hg.ff_triangles(ctx, grid, sd_dev, None, "f32c", out=out, out_type="c64",
                        pixels_per_thread=tuned_p)

    def barrier():
        if dist is not None:
            dist.barrier()

    for _ in range(max(3, args.warmup)):
        step()
    torch.cuda.synchronize()
    ctx.synchronize()

    peak_fp32, peak_sfu = hg.measure_peaks(ctx, sustained_ms=2000)
    peak_fp64 = hg.measure_peak_fp64(ctx)

    clk = Clocks(local)
    barrier()
    torch.cuda.synchronize()
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        step()
    e1.record(stream)
    torch.cuda.synchronize()
    barrier()
    clocks = clk.stop()
    ctx.synchronize()
    ms = max_over_ranks(e0.elapsed_time(e1), dist, dev)
    ms_step = ms / args.steps
    value = job_throughput(world, evals * args.steps, ms * 1e-3)

    # end to end through the reference-shaped C-ABI call with host (pinned) buffers
    e2e = None
    if not args.no_e2e:
        g = grid.read(qz_det=False, alpha=False)
        h_sd = torch.tensor(sd).pin_memory()
        h_qx = torch.tensor(g["qx"]).pin_memory()
        h_qy = torch.tensor(g["qy"]).pin_memory()
        h_qz = torch.tensor(g["qz_ext"]).pin_memory()
        h_out = torch.empty(4 * n, dtype=torch.complex128).pin_memory()
        hg.ff_triangles_arrays(ctx, h_sd, h_qx, h_qy, h_qz, None, "f32c", out=h_out)
        torch.cuda.synchronize()
        k = max(1, min(args.steps, 3))
        b0 = torch.cuda.Event(enable_timing=True)
        b1 = torch.cuda.Event(enable_timing=True)
        b0.record(stream)
        for _ in range(k):
            hg.ff_triangles_arrays(ctx, h_sd, h_qx, h_qy, h_qz, None, "f32c", out=h_out)
        b1.record(stream)
        torch.cuda.synchronize()
        mse = max_over_ranks(b0.elapsed_time(b1) / k, dist, dev)
        e2e = {"value": job_throughput(world, evals, mse * 1e-3), "unit": "evals/s",
               "h2d_bytes_per_step": int(sd.nbytes + 2 * 8 * n + 16 * 4 * n),
               "d2h_bytes_per_step": int(16 * 4 * n), "ms_per_step": mse,
               "path": "hgx_ff_triangles (reference-shaped, host buffers, complex128 out)"}

    # FP64 plain kernel on the same inputs (the denominator of the FP32 speed-up)
    f64 = None
    if not args.no_f64:
        out64 = torch.empty(4 * n, dtype=torch.complex128, device=dev)
        hg.ff_triangles(ctx, grid, sd_dev, None, "f64", out=out64, out_type="c128")
        torch.cuda.synchronize()
        a0 = torch.cuda.Event(enable_timing=True)
        a1 = torch.cuda.Event(enable_timing=True)
        reps64 = 2
        a0.record(stream)
        for _ in range(reps64):
            hg.ff_triangles(ctx, grid, sd_dev, None, "f64", out=out64, out_type="c128")
        a1.record(stream)
        torch.cuda.synchronize()
        ms64 = a0.elapsed_time(a1) / reps64
        # accuracy of the timed FP32 output against the FP64 kernel (norm-wise)
        d = (out.to(torch.complex128) - out64)
        relerr = float(torch.linalg.vector_norm(d) / torch.linalg.vector_norm(out64))
        # pointwise: |F32C - F64| / |F64| on the q-points whose |F|^2 is at least a fraction of
        # the largest (the weak q-points of a DWBA image carry the smallest amplitudes)
        a64 = out64.abs()
        rel = d.abs() / a64.clamp_min(1e-300)
        pw = {}
        for frac in (1e-6, 1e-3):
            r = rel[a64 * a64 >= frac * float((a64 * a64).max())]
            q = torch.quantile(r[torch.randperm(r.numel(), device=r.device)[:1 << 20]].float(),
                               torch.tensor([0.5, 0.99], device=r.device))
            pw[f"intensity_ge_{frac:g}_of_max"] = {"q_points": int(r.numel()), "median": float(q[0]),
                                                   "p99": float(q[1]), "max": float(r.max())}
        v64 = evals / (ms64 * 1e-3)
        f64 = {"value": v64, "unit": "evals/s", "ms_per_step": ms64, "launches_timed": reps64,
               "fp32c_speedup": (value / world) / v64, "fp32c_rel_err_vs_fp64": relerr,
               "fp32c_pointwise_rel_err": pw}
        del out64, a64, rel

    fit = None
    if not args.no_fitting and world == 1:  # the single-GPU legs stay out of scaling runs
        fit = fitting_bench(ctx, torch, dev, stream)
        bt = fit["batch_256_rois"]
        bt["roofline"] = roofline_of(
            "fp32", CYL_F32C_FP32_FLOP_PER_PIXEL, float(bt["pixels"]), bt["ms_per_batch"] * 1e-3, peak_fp32,
            "ROI pixel", "ncu executed FP32 FLOP of cyl_pixels_f32c_kernel (plus 60 FP64 per pixel); issue-"
            "bound with no pipe above 31% in ncu; the time is the whole graph (set-up, pixel pass, sums)")
        bt["fp64_adjoint"]["roofline"] = roofline_of(
            "fp64", CYL_F64_FLOP_PER_PIXEL, float(bt["pixels"]), bt["fp64_adjoint"]["ms_per_batch"] * 1e-3,
            peak_fp64, "ROI pixel", "ncu executed FP64 FLOP of cyl_pixels_kernel<double>")
        fit["mesh_vertices_2048sq"] = mesh_grad_bench(ctx, grid)
        mv = fit["mesh_vertices_2048sq"]
        mv["roofline"] = roofline_of(
            "fp32", MESH_FWD_FLOP_PER_PIXEL_TRI + MESH_BWD_FLOP_PER_PIXEL_TRI, float(n) * mv["triangles"],
            mv["s_per_eval"], peak_fp32, "(pixel, triangle): forward 40 + backward 80",
            "the expressions as written; ncu counts 82.5 executed in the backward")

    exact = None
    if not args.no_exact and world == 1:
        exact = exact_bench(ctx, torch, stream, sd)
        exact["roofline"] = roofline_of("fp64", EXACT_FP64_FLOP_PER_EVAL, exact["value"], 1.0, peak_fp64,
                                        "(q-point, triangle)", "ncu executed FP64 FLOP, 512^2 launch")

    hig = None
    if not args.no_hig and rank == 0 and world == 1:
        hig = hig_bench(ctx)
        pg = float(hig["pixels"]) * hig["grains"]
        hig["roofline"] = roofline_of("fp64", GRAIN_FP64_FLOP_PER_PIXEL_GRAIN, pg,
                                      hig["ms_per_simulation"] * 1e-3, peak_fp64, "(pixel, grain)",
                                      "ncu executed FP64 FLOP of grain_dwba_kernel on this description; "
                                      "the time is the whole simulation")
        if "f32c" in hig:
            hig["f32c"]["roofline"] = roofline_of(
                "fp32", GRAIN_F32C_FP32_FLOP_PER_PIXEL_GRAIN, pg, hig["f32c"]["ms_per_simulation"] * 1e-3,
                peak_fp32, "(pixel, grain)", "ncu executed FP32 FLOP of grain_dwba_f32c_kernel (plus 367 "
                "FP64 per unit); issue-bound (80% in ncu; XU 26%)")

    cfg1 = None
    if not args.no_config1 and rank == 0 and world == 1:
        cfg1 = config1_bench(ctx, cpu=not args.no_cpu_baseline)
        cfg1["population_512sq"] = population_bench(ctx)
        npx1 = float(cfg1["pixels"])
        t32, t64 = cfg1["f32c"]["ms"] * 1e-3, cfg1["f64"]["ms"] * 1e-3
        r32 = roofline_of("fp32", CFG1_F32C_FP32_FLOP_PER_PIXEL, npx1, t32, peak_fp32, "pixel",
                          "ncu executed FP32 FLOP of grain_dwba_f32c_kernel (plus 554 FP64 per pixel); "
                          "the time is the whole simulation (set-up, Fresnel coefficients, grain kernel, sums)")
        xu = CFG1_F32C_XU_PER_PIXEL * npx1 / t32 / 1e9
        r32["sfu"] = {"ops_per_unit": CFG1_F32C_XU_PER_PIXEL, "achieved_gops": xu, "peak_gops": peak_sfu,
                      "frac": xu / peak_sfu, "note": "XU-pipe thread operations (transcendentals and "
                      "conversions); 29% busy in ncu, the kernel issue-bound (81%)"}
        cfg1["f32c"]["roofline"] = r32
        cfg1["f64"]["roofline"] = roofline_of("fp64", CFG1_F64_FLOP_PER_PIXEL, npx1, t64, peak_fp64, "pixel",
                                              "ncu executed FP64 FLOP of grain_dwba_kernel; the time is "
                                              "the whole simulation")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        g = grid.read(qz_det=False, alpha=False)
        rate, threads, kind, desc = cpu_sample_rate(sd, g["qx"], g["qy"], g["qz_ext"])
        cpu = {"value": rate, "unit": "evals/s", "cores": threads, "kind": kind, "sample": desc}

    if rank == 0:
        flop = FLOP_PER_PIXEL_TRI * n * ntri
        achieved = flop / (ms_step * 1e-3) / 1e12
        sfu_rate = SFU_PER_PIXEL_TRI * n * ntri / (ms_step * 1e-3) / 1e9
        line = {
            "metric": "q.triangle evals/s", "value": value, "unit": "evals/s",
            "n_gpus": world, "steps": args.steps, "warmup": max(3, args.warmup),
            "ms_per_step": ms_step, "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32 (compensated; FP64 q-grid/epilogue)",
            "data": "synthetic (seeded star mesh, 50,000 triangles)",
            "config": {"workload": "mesh50k-dwba-2048sq: numeric FF, 50,000-triangle star "
                                   "mesh, 2048x2048 detector, 4 DWBA blocks",
                       "triangles": ntri, "grid": [NCOL, NROW], "blocks": 4,
                       "evals_per_step": evals, "parallelism": f"replicas x{world}",
                       "l2": "inputs larger than L2 (q-grid 332 MB)",
                       "launch_shape": {"pixels_per_thread": tuned_p,
                                        "kernel": "packed FP32x2" if tuned_p < 0 else "scalar",
                                        "autotuner_ms_8192_triangles":
                                            {str(k): v for k, v in tune_times.items()}}},
            "roofline": {"bound": "fp32", "achieved": achieved, "peak": peak_fp32,
                         "unit": "TFLOP/s", "frac": achieved / peak_fp32,
                         "traffic": TRAFFIC_BYTES_PER_LAUNCH,
                         "traffic_source": TRAFFIC_SOURCE,
                         "peak_source": "hgx_measure_peaks FFMA probe, sustained 2 s, same GPU",
                         "flop_per_pixel_triangle": FLOP_PER_PIXEL_TRI,
                         "sfu": {"achieved_gops": sfu_rate, "peak_gops": peak_sfu,
                                 "frac": sfu_rate / peak_sfu},
                         "hbm_view": hbm_view(ms_step)},
            "peaks": {"fp32_tflops": peak_fp32, "fp64_tflops": peak_fp64, "sfu_gops": peak_sfu,
                      "source": "the library's probes on this GPU (FFMA sustained 2 s, DFMA burst, __sinf)"},
            "cpu_baseline": cpu, "e2e": e2e, "fp64_plain": f64, "fitting": fit,
            "exact_triangle": exact, "hig_simulation": hig, "config1_dwba_1024sq": cfg1,
            "gpu_launches": HGX_LAUNCHES_PER_STEP * args.steps,
            "library_launches": {"cub_radix_sort": CUB_LAUNCHES_PER_STEP * args.steps},
            "clocks": clocks,
        }
        print(json.dumps(line), flush=True)
    grid.close()
    ctx.close()
    if dist is not None:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

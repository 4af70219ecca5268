"""Benchmark: parallel-beam SIRT / MLEM on one B200 (batched vs plain).

Workload (the 512x512x256 parallel-beam SIRT/MLEM configuration): a seeded
phantom of 20 random ellipses per slice on a 512x512x256 grid, projected
noiselessly at 720 angles in [0, pi) onto 768 detector columns x 256 rows
(log data), then reconstructed on the grid the reference derives from that
detector, 768x768x256.  A step is one SIRT iteration over all 256 slices:
forward projection with the residual update fused in, back projection with
the volume update fused in, captured once as a CUDA graph.  `value` is
iterations/s of that batched form with the data already on the GPU;
`plain_iter_per_s` is the one-slice-per-launch, host-driven form (measured
on a subset of slices and scaled, see its sample key); `e2e` runs the
reference-facing C-ABI call (host buffers, copies included).

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]

Under torchrun each rank solves its own 256-slice slab (weak scaling, no
collective on the data path); the time is the maximum over ranks.
"""
from __future__ import annotations

import argparse
import json
import math
import os
import statistics
import subprocess
import sys
import tempfile
import time

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, os.path.join(ROOT, "ccpi-reconstruction_b200"))

METRIC = "CGLS iter/s & projector rays/s on B200, batched vs plain, at ≤1e-4 rel L2 err"
NA, NV, NH = 720, 256, 768
PHANTOM = (512, 512, 256)
WORKLOAD = ("parallel-beam SIRT, 512x512x256 ellipse phantom (20/slice) projected at 720 "
            "angles onto 768x256 detector, reconstructed on the 768x768x256 grid, all 256 "
            "slices per step")
# --small: the same workload shrunk for profiler captures (still larger
# than L2: 189 MB sinogram, 268 MB volume)
SMALL = dict(NA=360, NV=256, NH=512, PHANTOM=(344, 344, 256),
             WORKLOAD="parallel-beam SIRT, 344x344x256 phantom, 360 angles, 512x256 detector, "
                      "512x512x256 grid (profiling size)")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="b200", choices=["b200", "reference"])
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--small", action="store_true", help="profiling-size workload")
    args = ap.parse_args()
    if args.small:
        g = globals()
        for k, v in SMALL.items():
            g[k] = v
    return args


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


# ------------------------------------------------------------------ data
def phantom(torch, dev, seed):
    """20 random ellipses per slice: centres uniform in the inner 80% of the
    slice, semi-axes 20-160 px, random rotation, densities U[0.1, 1],
    overlapping densities added (draw order: centres, axes, rotation,
    density, per slice)."""
    import numpy as np
    nx, ny, nz = PHANTOM
    rng = np.random.default_rng(seed)
    ne = 20
    cen = rng.uniform(-0.4, 0.4, (nz, ne, 2)) * nx
    ax = rng.uniform(20.0, 160.0, (nz, ne, 2))
    rot = rng.uniform(0.0, math.pi, (nz, ne))
    den = rng.uniform(0.1, 1.0, (nz, ne))
    c = torch.arange(nx, device=dev, dtype=torch.float32) + 0.5 - nx / 2
    X = c.view(nx, 1).expand(nx, ny)
    Y = c.view(1, ny).expand(nx, ny)
    vol = torch.zeros((nx, ny, nz), device=dev, dtype=torch.float32)
    for k in range(nz):
        acc = torch.zeros((nx, ny), device=dev)
        for e in range(ne):
            ct, st = math.cos(rot[k, e]), math.sin(rot[k, e])
            xr = (X - cen[k, e, 0]) * ct + (Y - cen[k, e, 1]) * st
            yr = -(X - cen[k, e, 0]) * st + (Y - cen[k, e, 1]) * ct
            acc += ((xr / ax[k, e, 0]) ** 2 + (yr / ax[k, e, 1]) ** 2 <= 1.0).float() * float(den[k, e])
        vol[:, :, k] = acc
    return vol


def make_problem(torch, dev, seed):
    """Returns (api plan, log sinogram (na, nh, nv) on the device, mu)."""
    import numpy as np
    from ccpi.reconstruction.device import Plan
    from ccpi.reconstruction.parallelbeam import alg
    ang = (math.pi * (np.linspace(0.0, 180.0, NA, endpoint=False).astype(np.float32)
                      .astype(np.float64) / 180.0))
    h = np.arange(NH) - (NH - 1) / 2.0
    v = np.arange(NV) - (NV - 1) / 2.0
    nx, ny, nz = PHANTOM
    ph_plan = Plan("parallel", ang, h, v, (-nx / 2, -ny / 2, -nz / 2), (1.0, 1.0, 1.0), PHANTOM)
    sino = ph_plan.forward(phantom(torch, dev, seed))
    mu = 3.0 / float(sino.max())  # max line integral 3
    sino.mul_(mu)
    gx, gy, gz, nvp, _ = alg.grid(NA, NV, NH, 0.0, 1)
    plan = Plan("parallel", ang, h, v, (-gx / 2, -gy / 2, -gz / 2), (1.0, 1.0, 1.0), (gx, gy, gz))
    ph_plan.close()
    return plan, sino, mu


# ----------------------------------------------------------------- clocks
class Clocks:
    def __init__(self, index):
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
             "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
             "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--id={index}", f"--query-gpu={q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        out = {"sm_mhz": None, "sm_max_mhz": None, "reasons": []}
        if self.p is None:
            return out
        self.p.terminate()
        self.p.wait()
        self.f.flush()
        rows = []
        with open(self.f.name) as f:
            for line in f:
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9:
                    rows.append(parts)
        os.unlink(self.f.name)
        if not rows:
            return out
        sm = [float(r[1]) for r in rows if r[1].replace(".", "").isdigit()]
        out["sm_mhz"] = statistics.median(sm) if sm else None
        out["sm_max_mhz"] = float(rows[0][2]) if rows[0][2].replace(".", "").isdigit() else None
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        seen = set()
        for r in rows:
            for n, val in zip(names, r[5:9]):
                if val.lower() == "active":
                    seen.add(n)
        out["reasons"] = sorted(seen)
        out["samples"] = len(rows)
        return out


# ------------------------------------------------------------ reference CPU
def cpu_reference_sample(sino_np_log):
    """The reference's own SIRT (compiled from its sources, oracle/_ref) on a
    bounded sample of the workload: 24 of the 720 angles x 4 of the 256
    slices x all 768 columns, 1 and 2 iterations; the difference is one
    iteration of the sample, scaled by 30 x 64 to the full workload."""
    import numpy as np
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.reference_available():
        return None
    idx = np.arange(0, NA, max(NA // 24, 1))[:24]
    rows = slice(NV // 2 - 2, NV // 2 + 2)
    ang = np.linspace(0.0, 180.0, NA, endpoint=False).astype(np.float32)[idx]
    pix = np.ascontiguousarray(np.transpose(sino_np_log[idx][:, :, rows], (0, 2, 1)))
    threads = os.cpu_count() or 1
    times = []
    for it in (1, 2):
        t0 = time.perf_counter()
        with O.quiet():
            O.ref_pb_reconstruct(1, pix, ang, 0.0, 1, it, True, nthreads=threads)
        times.append(time.perf_counter() - t0)
    t_iter = max(times[1] - times[0], 1e-9) * (NA / 24) * (NV / 4)
    return {"value": 1.0 / t_iter, "unit": "iter/s", "cores": threads, "kind": "reference",
            "sample": "reference SIRT (Core/src, -O2 -fopenmp) on 24 of 720 angles x 4 of 256 "
                      "slices x 768 columns; t(2 iter) - t(1 iter) scaled x30 x64 to the "
                      "full workload"}


def run_reference(args):
    """--impl reference: the reference's CPU path, each step a bounded
    sample of the workload (see cpu_reference_sample), on all host cores."""
    import numpy as np
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    if not O.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libccpi_ref.so not built"}))
        return
    rng = np.random.default_rng(2)
    sino = rng.random((NA, NH, NV)).astype(np.float32) * 2.0
    vals = []
    for i in range(args.warmup + args.steps):
        cb = cpu_reference_sample(sino)
        if i >= args.warmup:
            vals.append(cb["value"])
    v = statistics.median(vals)
    cb["value"] = v
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "iter/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": WORKLOAD},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


# -------------------------------------------------------------------- main
def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    import ctypes

    import numpy as np
    import torch
    import torch.distributed as dist

    from ccpi.reconstruction import _native as N
    from ccpi.reconstruction.device import Plan, Session

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    dev = torch.device("cuda", local)
    torch.cuda.set_device(dev)
    if world > 1:
        import datetime
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                device_id=dev)

    from ccpi.reconstruction import distributed as D

    def barrier():
        D.barrier()

    def max_over_ranks(x):
        return D.max_over_ranks(x, device=dev)

    plan, sino, mu = make_problem(torch, dev, seed=2 + rank)
    V = plan.shape[0] * plan.shape[1] * plan.shape[2]
    P = NA * NH * NV
    stream = torch.cuda.current_stream(dev)

    # ---- batched, graph-captured SIRT (the headline)
    x = torch.zeros(plan.shape, device=dev)
    sess = Session(plan, N.SIRT, sino, x, args.warmup + args.steps)
    sess.run(args.warmup)
    torch.cuda.synchronize()
    barrier()
    clocks = Clocks(local)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    torch.cuda.nvtx.range_push("sirt_timed")  # lets a profiler select the timed launches
    sess.run(args.steps)
    torch.cuda.nvtx.range_pop()
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_sirt = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
    sess.finish()
    sess.close()
    barrier()

    # ---- MLEM, same form
    xm = torch.zeros(plan.shape, device=dev)
    sm = Session(plan, N.MLEM, sino, xm, args.warmup + args.steps)
    sm.run(args.warmup)
    torch.cuda.synchronize()
    barrier()
    e0.record(stream)
    sm.run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    t_mlem = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
    sm.finish()
    sm.close()
    del xm

    # ---- dominant kernel: forward vs back projection, CUDA events
    tmp_p = torch.empty_like(sino)
    tmp_v = torch.empty(plan.shape, device=dev)
    for _ in range(2):
        plan.forward(x, tmp_p)
        plan.backward(sino, tmp_v)
    torch.cuda.synchronize()
    reps = 3
    e0.record(stream)
    for _ in range(reps):
        plan.forward(x, tmp_p)
    e1.record(stream)
    torch.cuda.synchronize()
    t_fp = e0.elapsed_time(e1) / 1000.0 / reps
    e0.record(stream)
    for _ in range(reps):
        plan.backward(sino, tmp_v)
    e1.record(stream)
    torch.cuda.synchronize()
    t_bp = e0.elapsed_time(e1) / 1000.0 / reps
    del tmp_p, tmp_v

    # ---- plain: one slice per launch sequence, host-driven iterations
    plain = None
    if not args.no_plain:
        from ccpi.reconstruction.parallelbeam import alg
        gx, gy, gz, _, _ = alg.grid(NA, NV, NH, 0.0, 1)
        ang = plan._arrays[0]
        h = np.arange(NH) - (NH - 1) / 2.0
        p1 = Plan("parallel", ang, h, np.array([0.0]), (-gx / 2, -gy / 2, -0.5), (1.0, 1.0, 1.0),
                  (gx, gy, 1))
        n_slices, n_it = 4, 2
        xs = torch.zeros((gx, gy, 1), device=dev)
        sk = sino[:, :, :1].contiguous()
        s1 = Session(p1, N.SIRT, sk, xs, 1, plain=True)
        s1.run(1)
        s1.finish()
        s1.close()
        torch.cuda.synchronize()
        t_run = 0.0
        for k in range(n_slices):
            sk = sino[:, :, NV // 2 + k:NV // 2 + k + 1].contiguous()
            xs.zero_()
            s1 = Session(p1, N.SIRT, sk, xs, n_it, plain=True)
            torch.cuda.synchronize()
            t0 = time.perf_counter()
            s1.run(n_it)
            torch.cuda.synchronize()
            t_run += time.perf_counter() - t0
            s1.finish()
            s1.close()
        t_slice_it = t_run / (n_slices * n_it)
        plain = {"iter_per_s": 1.0 / (t_slice_it * NV),
                 "sample": f"{n_slices} single-slice SIRT solves x {n_it} host-driven "
                           f"iterations each (set-up excluded); time per slice-iteration "
                           f"x 256 slices"}
        p1.close()

    # ---- e2e through the reference-facing C ABI with pinned host buffers
    e2e_it = args.steps
    host_in = torch.empty((NA, NV, NH), dtype=torch.float32, pin_memory=True)
    host_in.copy_(sino.permute(0, 2, 1).cpu())
    ang32 = np.linspace(0.0, 180.0, NA, endpoint=False).astype(np.float32)
    gx, gy, gz = plan.shape
    host_out = torch.empty((gx, gy, gz), dtype=torch.float32, pin_memory=True)
    barrier()
    t0 = time.perf_counter()
    rc = N.lib.ccpi_pb_reconstruct(N.SIRT, host_in.numpy(), NA, NV, NH, ang32, 0.0, 1, e2e_it, 1,
                                   1, 0.0, None, None, host_out.numpy())
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    N.check(rc, "ccpi_pb_reconstruct")

    # ---- CPU baseline (rank 0, N = 1 only)
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = cpu_reference_sample(sino.cpu().numpy())

    if rank == 0:
        peak, peak_kind = load_peaks()
        value = world * args.steps / t_sirt
        alg_bytes = 4.0 * (V + P)  # one projection: read the input, write the output
        t_dom, dom = (t_bp, "pb_bp (back projection)") if t_bp >= t_fp else (t_fp, "pb_fp (forward projection)")
        achieved = alg_bytes / t_dom / 1e9
        rays = P / t_fp
        line = {
            "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * t_sirt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "solver": "SIRT", "grid": list(plan.shape),
                       "angles": NA, "detector": [NH, NV], "mu": mu,
                       "l2": "inputs larger than L2 (sinogram 566 MB, volume 604 MB)",
                       "form": "batched: all slices per launch, one CUDA graph per iteration"},
            "mlem_iter_per_s": world * args.steps / t_mlem,
            "fp_ms": 1000.0 * t_fp, "bp_ms": 1000.0 * t_bp,
            "projector_rays_per_s": {"forward": rays, "backward": P / t_bp},
            "plain_iter_per_s": plain["iter_per_s"] if plain else None,
            "batched_over_plain": (value / world) / plain["iter_per_s"] if plain else None,
            "plain_sample": plain["sample"] if plain else None,
            "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": peak,
                         "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind,
                         "algorithmic_bytes_per_launch": alg_bytes, "traffic": None},
            "e2e": {"value": world * e2e_it / t_e2e, "unit": "iter/s",
                    "h2d_bytes_per_step": host_in.numel() * 4 / e2e_it,
                    "d2h_bytes_per_step": host_out.numel() * 4 / e2e_it,
                    "call": "ccpi_pb_reconstruct(SIRT, %d iterations), pinned host buffers" % e2e_it},
            "gpu_launches": 2 * args.steps,
            "clocks": clk,
            "cpu_baseline": cpu,
        }
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark: CGLS iterations/s on one B200 (graph-captured vs plain).

Headline workload (the 512^3 cone-beam CGLS configuration): 40 seeded
ellipsoids (semi-axes 10-120 voxels, densities U[0.1, 1]) in a 512^3 grid of
1 mm voxels, projected at 720 angles over [0, 2 pi) onto a 768 x 768
detector of 0.8 mm pixels (source and detector 500 mm from the axis),
Poisson noise at 5e3 photons per ray, then CGLS on the explicit 512^3 grid.
A step is one CGLS iteration: forward projection with the FP64 sum of
squares fused in, the residual update, back projection with its FP64 sum of
squares fused in, the x/d update; the iteration is captured once as a CUDA
graph.  `value` is iterations/s with the data resident on the GPU;
`plain_iter_per_s` the same iterations launched from the host with the step
scalars read back every iteration; `e2e` the host-buffer C-ABI call
ccpi_reconstruct (copies and set-up included); `cpu_baseline` the
reference's own cone CGLS on an angle sample of the same workload.

`parallel_sirt` carries the 768x768x256 parallel-beam SIRT/MLEM
configuration (720 angles, 768 x 256 detector, all 256 slices per launch)
with its own roofline, plain/batched ratio, e2e and CPU baseline.

  python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
  python bench.py --workload {sirt,uneven,autograd}   # one line each

Under torchrun each rank solves its own problem (cone beam: replicas; the
parallel-beam part: its own 256-slice slab), no collective on the data
path; the time is the maximum over ranks.
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
# cone-beam CGLS workload
CN, CNA, CND, CPIX, CS2O, CO2D = 512, 720, 768, 0.8, 500.0, 500.0
CONE_WORKLOAD = ("cone-beam CGLS, 512^3 ellipsoid phantom (40), 720 angles over 2 pi, "
                 "768x768 detector at 0.8 mm, source/detector 500 mm, Poisson 5e3, explicit "
                 "512^3 grid of 1 mm voxels")
CONE_SAMPLE_ANGLES = 48  # angle sample of the CPU baselines: divides 720, a multiple of 16 cores
# parallel-beam SIRT/MLEM workload
NA, NV, NH = 720, 256, 768
PHANTOM = (512, 512, 256)
WORKLOAD = ("parallel-beam SIRT, 512x512x256 ellipse phantom (20/slice) projected at 720 "
            "angles onto 768x256 detector, reconstructed on the 768x768x256 grid, all 256 "
            "slices per step")
# --small: the parallel workload shrunk for profiler captures (still larger
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
    ap.add_argument("--no-fp64", action="store_true",
                    help="skip the FP64-oracle check on the 1/4-scale cone copy")
    ap.add_argument("--no-parallel", action="store_true",
                    help="skip the parallel-beam SIRT/MLEM part of the default line")
    ap.add_argument("--small", action="store_true", help="profiling-size parallel workload")
    ap.add_argument("--workload", default="cone-cgls",
                    choices=["cone-cgls", "sirt", "uneven", "autograd", "cone-projectors"],
                    help="cone-cgls: the default line; the others print their own line")
    ap.add_argument("--cone-n", type=int, default=CN,
                    help="cone grid edge (512: the CGLS workload; 256: 360 angles onto a 384^2 "
                         "detector at 1.6 mm, 2 mm voxels, for profiler captures)")
    ap.add_argument("--cone-bp", default="auto", choices=["auto", "gather", "scatter"],
                    help="cone back projector: auto (ccpi_plan_autotune times both, outside "
                         "the timed region), the voxel gather or the ray-driven scatter")
    args = ap.parse_args()
    if args.small:
        g = globals()
        for k, v in SMALL.items():
            g[k] = v
    return args


def load_traffic(kernel):
    """DRAM bytes per launch of `kernel` on the full-size workload, from one
    ncu capture of the same command (1-pass metrics), kept in profiles/."""
    name = {"pb_fp": "pb_traffic_768x768x256.json", "pb_bp": "pb_traffic_768x768x256.json",
            "cb_bp_gather": "cb_traffic_512cube.json", "cb_bp_scatter": "cb_traffic_512cube.json",
            "cb_fp": "cb_traffic_512cube.json"}.get(kernel)
    if name is None or (kernel.startswith("pb") and globals().get("NH") != 768):
        return None
    try:
        with open(os.path.join(ROOT, "profiles", name)) as f:
            return float(json.load(f)["kernels"][kernel]["dram_bytes_per_launch"])
    except Exception:
        return None


def pick_cone_bp(plan, choice):
    """Set the cone plan's back projector as --cone-bp asks; returns
    (kernel name, seconds the autotuner took or 0)."""
    t = 0.0
    if choice == "auto":
        t0 = time.perf_counter()
        scatter = plan.autotune()[1] == 1
        t = time.perf_counter() - t0
    else:
        scatter = choice == "scatter"
        plan.set_cone_backprojector(1 if scatter else 0)
    return ("cb_bp_scatter" if scatter else "cb_bp_gather"), t


def load_peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def oracle():
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    return O


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


def ellipsoid_phantom(n, count, axes, seed):
    """numpy float32 n^3 volume: the sum of `count` seeded ellipsoids with
    centres in the inner 60 %, semi-axes U[axes] voxels, a random
    orientation (Q of the QR of a normal 3x3 draw) and densities U[0.1, 1]
    (draw order: centre, axes, rotation, density, per ellipsoid).  Each
    ellipsoid is evaluated inside its bounding box only."""
    import numpy as np
    rng = np.random.default_rng(seed)
    vol = np.zeros((n, n, n), np.float32)
    c = (np.arange(n, dtype=np.float32) + np.float32(0.5) - np.float32(n / 2))
    for _ in range(count):
        cen = rng.uniform(-0.3, 0.3, 3) * n
        ax = rng.uniform(axes[0], axes[1], 3)
        q, _r = np.linalg.qr(rng.standard_normal((3, 3)))
        den = np.float32(rng.uniform(0.1, 1.0))
        r = float(ax.max()) + 1.0
        lo = [max(int(math.floor(cen[i] + n / 2 - r)), 0) for i in range(3)]
        hi = [min(int(math.ceil(cen[i] + n / 2 + r)) + 1, n) for i in range(3)]
        if any(lo[i] >= hi[i] for i in range(3)):
            continue
        dx = (c[lo[0]:hi[0]] - np.float32(cen[0]))[:, None, None]
        dy = (c[lo[1]:hi[1]] - np.float32(cen[1]))[None, :, None]
        dz = (c[lo[2]:hi[2]] - np.float32(cen[2]))[None, None, :]
        acc = None
        for k in range(3):
            u = (dx * np.float32(q[0, k]) + dy * np.float32(q[1, k]) + dz * np.float32(q[2, k])) \
                / np.float32(ax[k])
            acc = u * u if acc is None else acc + u * u
        vol[lo[0]:hi[0], lo[1]:hi[1], lo[2]:hi[2]] += (acc <= 1.0).astype(np.float32) * den
    return vol


def cone_geometry(n):
    """(grid edge, voxel mm, angles, detector edge, pixel mm) of the cone
    workload (n = 512) or its 256^3 profiling copy (360 angles onto a 384^2
    detector at 1.6 mm, 2 mm voxels: the same voxel shadow in pixels)."""
    return (CN, 1.0, CNA, CND, CPIX) if n == CN else (n, 2.0 * 256 / n, 360, 384, 1.6)


def cone_angles(count=CNA, every=1):
    import numpy as np
    return (np.arange(0, CNA, every)[:count]) * (2.0 * math.pi / CNA)


def cone_detector():
    import numpy as np
    d = (np.arange(CND) - (CND - 1) / 2.0) * CPIX
    return d, d.copy()


def poisson_log_torch(torch, clean, mu, i0, seed):
    gen = torch.Generator(device=clean.device).manual_seed(seed)
    counts = torch.poisson(i0 * torch.exp(-mu * clean), generator=gen)
    return -torch.log(torch.clamp(counts, min=1.0) / i0)


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


def cuda_time(torch, fn, reps=1):
    """Seconds per call of fn on torch's current stream (CUDA events)."""
    s = torch.cuda.current_stream()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(s)
    for _ in range(reps):
        fn()
    e1.record(s)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1000.0 / reps


# ------------------------------------------------------------ reference CPU
def cone_reference_sample(vol_np, n_angles, niters, threads):
    """The reference's own cone CGLS (cgls_3d over cone_beam::f2D/b2D,
    compiled from its sources into oracle/_ref) on the full 512^3 grid and
    768^2 detector with `n_angles` of the 720 angles (evenly spread).  The
    sample's log data is the reference's own projection of the phantom at
    those angles with the workload's noise model.  Returns the wall time of
    each call in `niters` (iteration counts; 0 = the set-up back projection
    alone)."""
    import numpy as np
    O = oracle()
    every = CNA // n_angles
    h, v = cone_detector()
    g = O.cone_geometry(CN, 1.0, n_angles, CND, CPIX, CS2O, CO2D)
    g.angles = cone_angles(n_angles, every)
    with O.quiet():
        clean = O.ref_forward(g, vol_np)
    mu = 3.0 / float(clean.max())
    rng = np.random.default_rng(3)
    counts = rng.poisson(5.0e3 * np.exp(-mu * clean.astype(np.float64)))
    sino = (-np.log(np.maximum(counts, 1) / 5.0e3)).astype(np.float32)
    del clean, counts
    out = []
    for it in niters:
        t0 = time.perf_counter()
        with O.quiet():
            O.ref_cb_solve_explicit(g, 0, sino, it, nthreads=threads)
        out.append(time.perf_counter() - t0)
    return out


def cone_cpu_baseline(vol_np):
    """One CGLS iteration of the reference on a 32-angle sample of the cone
    workload, t(2 iterations) - t(1 iteration), scaled by 720/32.  Every
    part of the reference's iteration but the vector updates (about 0.1 %
    of it) loops over angles: the forward projector's parallel loop
    (c2D.cpp:546) and the back projector's per-column ray search
    (c2D.cpp:831-936) and row loops."""
    O = oracle()
    if not O.reference_available():
        return None
    threads = os.cpu_count() or 1
    t1, t2 = cone_reference_sample(vol_np, CONE_SAMPLE_ANGLES, (1, 2), threads)
    t_iter = max(t2 - t1, 1e-9) * (CNA / CONE_SAMPLE_ANGLES)
    return {"value": 1.0 / t_iter, "unit": "iter/s", "cores": threads, "kind": "reference",
            "sample": f"reference cone CGLS (Core/src cgls_3d, -O2 -fopenmp, explicit 512^3 "
                      f"grid, 768^2 detector) on {CONE_SAMPLE_ANGLES} of the 720 angles; "
                      f"t(2 iterations) - t(1 iteration) = {t2 - t1:.2f} s, scaled x"
                      f"{CNA // CONE_SAMPLE_ANGLES} (time per iteration is linear in the "
                      f"angle count)"}


def run_reference(args):
    """--impl reference: the reference's CPU cone CGLS on the same workload,
    each step one iteration on a 32-angle sample scaled to the 720 angles
    (see cone_cpu_baseline), on all host cores.  W warm-up iterations run
    in one untimed call; the K timed iterations are t(K iterations) - t(0)
    (the set-up back projection alone)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    O = oracle()
    if not O.reference_available():
        print(json.dumps({"impl": "reference", "unavailable": "oracle/_ref/libccpi_ref.so not built"}))
        return
    threads = os.cpu_count() or 1
    vol = ellipsoid_phantom(CN, 40, (10.0, 120.0), seed=3)
    cone_reference_sample(vol, CONE_SAMPLE_ANGLES, (args.warmup,), threads)
    t0, tk = cone_reference_sample(vol, CONE_SAMPLE_ANGLES, (0, args.steps), threads)
    t_iter = max(tk - t0, 1e-9) / args.steps * (CNA / CONE_SAMPLE_ANGLES)
    v = 1.0 / t_iter
    cb = {"value": v, "unit": "iter/s", "cores": threads, "kind": "reference",
          "sample": f"reference cone CGLS on {CONE_SAMPLE_ANGLES} of 720 angles (every {CNA // CONE_SAMPLE_ANGLES}th), full 512^3 grid "
                    f"and 768^2 detector; (t({args.steps} iterations) - t(0)) / {args.steps} "
                    f"scaled x{CNA // CONE_SAMPLE_ANGLES}"}
    print(json.dumps({
        "impl": "reference", "metric": METRIC, "value": v, "unit": "iter/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 / v, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": {"workload": CONE_WORKLOAD},
        "cpu_baseline": cb,
        "e2e": {"value": v, "unit": "iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}))


def sirt_cpu_baseline(sino_np_log):
    """The reference's own SIRT (oracle/_ref) on 32 of the 720 angles with
    all 256 slices and 768 columns (the 768x768x256 grid),
    t(2 iterations) - t(1), scaled by 720/32 (the projectors loop over
    angles; every row and column is kept)."""
    import numpy as np
    O = oracle()
    if not O.reference_available():
        return None
    n = CONE_SAMPLE_ANGLES
    idx = np.arange(0, NA, NA // n)[:n]
    ang = np.linspace(0.0, 180.0, NA, endpoint=False).astype(np.float32)[idx]
    pix = np.ascontiguousarray(np.transpose(sino_np_log[idx], (0, 2, 1)))
    threads = os.cpu_count() or 1
    times = []
    for it in (1, 2):
        t0 = time.perf_counter()
        with O.quiet():
            O.ref_pb_reconstruct(1, pix, ang, 0.0, 1, it, True, nthreads=threads)
        times.append(time.perf_counter() - t0)
    t_iter = max(times[1] - times[0], 1e-9) * (NA / n)
    return {"value": 1.0 / t_iter, "unit": "iter/s", "cores": threads, "kind": "reference",
            "sample": f"reference SIRT (Core/src, -O2 -fopenmp) on {n} of 720 angles x all 256 "
                      f"slices x 768 columns of the phantom's sinogram; t(2 iter) - t(1 iter) "
                      f"= {times[1] - times[0]:.2f} s scaled x{NA // n}"}


# ----------------------------------------------------------- cone CGLS line
def cone_fp64_check(torch, dev):
    """GPU CGLS against the FP64 oracle on a 1/4-scale copy of the cone
    workload (128^3 at 4 mm, 180 angles, 192^2 detector at 3.2 mm, the same
    phantom recipe, Poisson 5e3), 30 iterations, with the reference's own
    FP32 CGLS beside it.  Also the distance after 10 iterations, before FP32
    CGLS loses conjugacy."""
    import numpy as np
    O = oracle()
    from ccpi.reconstruction.device import cone_plan
    n, na, nd = 128, 180, 192
    plan = cone_plan(n, 4.0, na, nd, 3.2, CS2O, CO2D)
    vol = torch.from_numpy(ellipsoid_phantom(n, 40, (2.5, 30.0), seed=3)).to(dev)
    clean = plan.forward(vol)
    sino = poisson_log_torch(torch, clean, 3.0 / float(clean.max()), 5.0e3, 3)
    g = O.cone_geometry(n, 4.0, na, nd, 3.2, CS2O, CO2D)
    s_np = sino.cpu().numpy()
    out = {"case": "128^3 at 4 mm, 180 angles, 192^2 detector at 3.2 mm, Poisson 5e3"}
    threads = os.cpu_count() or 1
    for it in (10, 30):
        x = torch.zeros(plan.shape, device=dev)
        plan.solve(0, sino, x, it)
        r64 = O.solve(g, 0, s_np.astype(np.float64), it, fp64=True)
        rel = lambda a: float(np.linalg.norm(a - r64) / np.linalg.norm(r64))  # noqa: E731
        d = {"rel_l2": rel(x.cpu().numpy().astype(np.float64))}
        if O.reference_available():
            with O.quiet():
                ref = O.ref_cb_solve_explicit(g, 0, s_np, it, nthreads=threads)
            d["reference_fp32_rel_l2"] = rel(ref.astype(np.float64))
        out[f"{it}_iterations"] = d
    plan.close()
    return out


def cone_line(args, torch, dev, world, rank, barrier, max_over_ranks):
    import numpy as np
    from ccpi.reconstruction import _native as N
    from ccpi.reconstruction.conebeam import alg as CA
    from ccpi.reconstruction.device import Session, cone_plan
    n, vs, na, nd, px = cone_geometry(args.cone_n)
    full = n == CN
    plan = cone_plan(n, vs, na, nd, px, CS2O, CO2D)
    bp_kernel, t_tune = pick_cone_bp(plan, args.cone_bp)
    vol_np = ellipsoid_phantom(n, 40, (10.0 * n / CN, 120.0 * n / CN), seed=3 + rank)
    clean = plan.forward(torch.from_numpy(vol_np).to(dev))
    mu = 3.0 / float(clean.max())
    sino = poisson_log_torch(torch, clean, mu, 5.0e3, 3 + rank)
    del clean
    V, P = n ** 3, na * nd * nd
    stream = torch.cuda.current_stream(dev)

    # ---- graph-captured CGLS (the headline), data resident
    x = torch.zeros(plan.shape, device=dev)
    sess = Session(plan, N.CGLS, sino, x, args.warmup + args.steps)
    sess.run(args.warmup)
    torch.cuda.synchronize()
    barrier()
    clocks = Clocks(torch.cuda.current_device())
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    sess.run(args.steps)
    e1.record(stream)
    torch.cuda.synchronize()
    clk = clocks.stop()
    t_cgls = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
    norms = sess.finish()
    sess.close()
    barrier()

    # ---- the projectors alone, CUDA events on the launching stream
    tmp_p = torch.empty_like(sino)
    t_fp = cuda_time(torch, lambda: plan.forward(x, tmp_p), 2)
    t_bp = cuda_time(torch, lambda: plan.backward(sino, x), 2)
    del tmp_p

    # ---- plain: host-driven iterations (each iteration's launches from the
    # host, step scalars read back every iteration)
    # (a session: set-up and workspace outside the timed region, W warm-up
    # iterations, then K iterations between CUDA events, as for `value`)
    plain = None
    if not args.no_plain:
        xp = torch.zeros(plan.shape, device=dev)
        ps = Session(plan, N.CGLS, sino, xp, args.warmup + args.steps, plain=True)
        ps.run(args.warmup)
        plain = cuda_time(torch, lambda: ps.run(args.steps)) / args.steps
        ps.finish()
        ps.close()
        del xp

    # ---- e2e: ccpi_reconstruct with pinned host buffers (upload, plan, set-up,
    # K iterations, download)
    host_s = torch.empty(sino.shape, dtype=torch.float32, pin_memory=True)
    host_s.copy_(sino)
    host_x = torch.empty(plan.shape, dtype=torch.float32, pin_memory=True)
    ang, h, v = (np.asarray(a, np.float64) for a in plan._arrays)
    geo = dict(source=(-CS2O, 0.0, 0.0), detector_x=CO2D, h_pixels=h, v_pixels=v, angles=ang,
               grid_offset=(-n * vs / 2.0,) * 3, voxel_size=(vs,) * 3, shape=(n,) * 3)
    del sino, x
    torch.cuda.empty_cache()

    # the call a user makes, with the back projector the autotuner chose for
    # the device plan (ccpi_reconstruct_flags, CCPI_RECON_CONE_SCATTER)
    e2e_form = "scatter" if bp_kernel == "cb_bp_scatter" else "gather"

    def e2e():
        out = CA.reconstruct_explicit("cgls", geo["source"], geo["detector_x"], geo["h_pixels"],
                                      geo["v_pixels"], geo["angles"], host_s.numpy(),
                                      geo["grid_offset"], geo["voxel_size"], geo["shape"],
                                      args.steps, backprojector=e2e_form)
        host_x.numpy()[...] = out
    barrier()
    t0 = time.perf_counter()
    e2e()
    t_e2e = max_over_ranks(time.perf_counter() - t0)
    plan.close()
    del host_s, host_x
    torch.cuda.empty_cache()

    fp64 = None
    cpu = None
    if rank == 0 and world == 1 and full:
        if not args.no_fp64:
            fp64 = cone_fp64_check(torch, dev)
        if not args.no_cpu:
            cpu = cone_cpu_baseline(vol_np)
    peak, peak_kind = load_peaks()
    bp_bytes = 4.0 * (V + P)
    it_bytes = 4.0 * (7 * V + 4 * P)
    traffic = load_traffic(bp_kernel)
    value = world * args.steps / t_cgls
    t_it = t_cgls / args.steps
    return {
        "metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1000.0 * t_it,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
        "data": "synthetic",
        "config": {"workload": CONE_WORKLOAD if full else
                   f"cone-beam CGLS, {n}^3 ellipsoid phantom, {na} angles, {nd}^2 detector "
                   f"(profiling size)", "solver": "CGLS", "grid": [n, n, n],
                   "angles": na, "detector": [nd, nd], "mu": mu,
                   "l2": "inputs larger than L2 (sinogram %.0f MB, volume %.0f MB)"
                         % (4.0 * P / 1e6, 4.0 * V / 1e6),
                   "form": "one CUDA graph per iteration",
                   "multi_gpu": "replicas: each rank solves its own problem"},
        "fp_ms": 1000.0 * t_fp, "bp_ms": 1000.0 * t_bp,
        "projector_rays_per_s": {"forward": P / t_fp, "backward": P / t_bp},
        "plain_iter_per_s": (1.0 / plain) if plain else None,
        "batched_over_plain": (plain / t_it) if plain else None,
        "plain_form": "host-driven iterations, step scalars read back each iteration",
        "roofline": {"bound": "hbm", "kernel": bp_kernel + " (back projection)",
                     "achieved": bp_bytes / t_bp / 1e9, "peak": peak, "unit": "GB/s",
                     "frac": bp_bytes / t_bp / 1e9 / peak, "peak_kind": peak_kind,
                     "algorithmic_bytes_per_launch": bp_bytes,
                     "traffic": traffic,
                     # DRAM bytes of one ncu capture of the same launch,
                     # moved in this run's launch time
                     "traffic_gbs": (traffic / t_bp / 1e9) if traffic else None,
                     "traffic_frac": (traffic / t_bp / 1e9 / peak) if traffic else None,
                     "algorithmic_over_traffic": (bp_bytes / traffic) if traffic else None},
        "iteration_roofline": {"achieved": it_bytes / t_it / 1e9, "unit": "GB/s",
                               "frac": it_bytes / t_it / 1e9 / peak,
                               "algorithmic_bytes_per_iteration": it_bytes},
        "e2e": {"value": world * args.steps / t_e2e, "unit": "iter/s",
                "h2d_bytes_per_step": 4.0 * P / args.steps,
                "d2h_bytes_per_step": 4.0 * V / args.steps,
                "call": "ccpi_reconstruct_flags(cone geometry, CGLS, %d iterations, %s back "
                        "projector), pinned host sinogram and volume; plan, upload, set-up and "
                        "download inside" % (args.steps, e2e_form)},
        # per iteration: forward, alpha, residual update, d_conv pre-scale,
        # back projection, beta, x/d update; the scatter's norm form adds a
        # sum-of-squares pass (its zero fill is a memset node)
        "gpu_launches": (8 if bp_kernel == "cb_bp_scatter" else 7) * args.steps,
        "back_projector": {"kernel": bp_kernel, "choice": args.cone_bp,
                           "autotune_seconds": t_tune},
        "clocks": clk,
        "residual_norms": [float(n_) for n_ in norms[-3:]],
        "fp64_oracle": fp64,
        "cpu_baseline": cpu,
    }


# ----------------------------------------------------- parallel SIRT part
def sirt_part(args, torch, dev, world, rank, barrier, max_over_ranks, full_line=False):
    """The 768x768x256 parallel-beam SIRT/MLEM workload: returns its numbers
    (the default line's `parallel_sirt`), or the old stand-alone line."""
    import ctypes

    import numpy as np
    from ccpi.reconstruction import _native as N
    from ccpi.reconstruction.device import Plan, Session

    plan, sino, mu = make_problem(torch, dev, seed=2 + rank)
    V = plan.shape[0] * plan.shape[1] * plan.shape[2]
    P = NA * NH * NV
    stream = torch.cuda.current_stream(dev)

    def timed_session(alg):
        x = torch.zeros(plan.shape, device=dev)
        s = Session(plan, alg, sino, x, args.warmup + args.steps)
        s.run(args.warmup)
        torch.cuda.synchronize()
        barrier()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        e0.record(stream)
        s.run(args.steps)
        e1.record(stream)
        torch.cuda.synchronize()
        t = max_over_ranks(e0.elapsed_time(e1) / 1000.0)
        s.finish()
        s.close()
        return t, x

    clocks = Clocks(torch.cuda.current_device()) if full_line else None
    t_sirt, x = timed_session(N.SIRT)
    clk = clocks.stop() if clocks else None
    t_mlem, _ = timed_session(N.MLEM)
    t_cg, _ = timed_session(N.CGLS) if full_line else (None, None)

    tmp_p = torch.empty_like(sino)
    tmp_v = torch.empty(plan.shape, device=dev)
    plan.forward(x, tmp_p)
    plan.backward(sino, tmp_v)
    t_fp = cuda_time(torch, lambda: plan.forward(x, tmp_p), 3)
    t_bp = cuda_time(torch, lambda: plan.backward(sino, tmp_v), 3)
    del tmp_p, tmp_v

    # the projectors' own ceiling: random whole-column reads from an
    # L2-resident 64 MiB set (ccpi_measure_gather).  Each ray-cell visit of
    # the FP (and each column-ray pair of the BP) moves one nz-float column;
    # for unit pixels and voxels one projection gathers
    # 4 V sum_a (|cos a| + |sin a|) bytes.
    gather_peak = np.zeros(1, np.float64)
    N.check(N.lib.ccpi_measure_gather(64 << 20, ctypes.c_void_p(stream.cuda_stream), gather_peak),
            "ccpi_measure_gather")
    ang_rad = np.asarray(plan._arrays[0], np.float64)
    gather_bytes = 4.0 * V * float(np.sum(np.abs(np.cos(ang_rad)) + np.abs(np.sin(ang_rad))))

    plain = None
    if not args.no_plain:
        from ccpi.reconstruction.parallelbeam import alg
        gx, gy, gz, _, _ = alg.grid(NA, NV, NH, 0.0, 1)
        h = np.arange(NH) - (NH - 1) / 2.0
        p1 = Plan("parallel", plan._arrays[0], h, np.array([0.0]), (-gx / 2, -gy / 2, -0.5),
                  (1.0, 1.0, 1.0), (gx, gy, 1))
        n_slices, n_it = 4, 2
        xs = torch.zeros((gx, gy, 1), device=dev)
        s1 = Session(p1, N.SIRT, sino[:, :, :1].contiguous(), xs, 1, plain=True)
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
        plain = 1.0 / (t_run / (n_slices * n_it) * NV)
        p1.close()

    # e2e through the reference-facing C ABI with pinned host buffers
    host_in = torch.empty((NA, NV, NH), dtype=torch.float32, pin_memory=True)
    host_in.copy_(sino.permute(0, 2, 1).cpu())
    ang32 = np.linspace(0.0, 180.0, NA, endpoint=False).astype(np.float32)
    host_out = torch.empty(plan.shape, dtype=torch.float32, pin_memory=True)
    N.check(N.lib.ccpi_pb_reconstruct(N.SIRT, host_in.numpy(), NA, NV, NH, ang32, 0.0, 1, 1, 1,
                                      1, 0.0, None, None, host_out.numpy()),
            "ccpi_pb_reconstruct")
    e2e_runs = []
    for _ in range(3):
        barrier()
        t0 = time.perf_counter()
        rc = N.lib.ccpi_pb_reconstruct(N.SIRT, host_in.numpy(), NA, NV, NH, ang32, 0.0, 1,
                                       args.steps, 1, 1, 0.0, None, None, host_out.numpy())
        e2e_runs.append(max_over_ranks(time.perf_counter() - t0))
        N.check(rc, "ccpi_pb_reconstruct")
    t_e2e = sorted(e2e_runs)[1]

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        cpu = sirt_cpu_baseline(sino.cpu().numpy())
    plan.close()
    del sino, x, host_in, host_out
    torch.cuda.empty_cache()

    peak, peak_kind = load_peaks()
    alg_bytes = 4.0 * (V + P)
    t_dom, dom = (t_bp, "pb_bp") if t_bp >= t_fp else (t_fp, "pb_fp")
    value = world * args.steps / t_sirt
    d = {
        "workload": WORKLOAD, "sirt_iter_per_s": value,
        "mlem_iter_per_s": world * args.steps / t_mlem,
        "fp_ms": 1000.0 * t_fp, "bp_ms": 1000.0 * t_bp,
        "projector_rays_per_s": {"forward": P / t_fp, "backward": P / t_bp},
        "plain_iter_per_s": plain, "batched_over_plain": (value / world) / plain if plain else None,
        "plain_sample": "4 single-slice SIRT solves x 2 host-driven iterations (set-up "
                        "excluded); time per slice-iteration x 256 slices",
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": alg_bytes / t_dom / 1e9,
                     "peak": peak, "unit": "GB/s", "frac": alg_bytes / t_dom / 1e9 / peak,
                     "peak_kind": peak_kind, "algorithmic_bytes_per_launch": alg_bytes,
                     "traffic": load_traffic(dom)},
        "gather_roofline": {
            "bound": "L2 -> SM gathers", "unit": "GB/s", "peak": float(gather_peak[0]),
            "peak_kind": "measured live: ccpi_measure_gather, random 1 KB columns, 64 MiB set, "
                         "grid %d CTAs" % (4 * torch.cuda.get_device_properties(dev).multi_processor_count),
            "bytes_per_launch": gather_bytes,
            "fp": {"achieved": gather_bytes / t_fp / 1e9,
                   "frac": gather_bytes / t_fp / 1e9 / float(gather_peak[0])},
            "bp": {"achieved": gather_bytes / t_bp / 1e9,
                   "frac": gather_bytes / t_bp / 1e9 / float(gather_peak[0])}},
        "e2e": {"value": world * args.steps / t_e2e, "unit": "iter/s",
                "h2d_bytes_per_step": NA * NV * NH * 4 / args.steps,
                "d2h_bytes_per_step": V * 4 / args.steps,
                "call": "ccpi_pb_reconstruct(SIRT, %d iterations), pinned host buffers; median "
                        "of 3 timed calls" % args.steps, "calls_s": e2e_runs},
        "cpu_baseline": cpu,
    }
    if not full_line:
        return d
    line = {"metric": METRIC, "value": value, "unit": "iter/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup,
            "ms_per_step": 1000.0 * t_sirt / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": WORKLOAD, "solver": "SIRT", "grid": list(plan.shape),
                       "angles": NA, "detector": [NH, NV], "mu": mu,
                       "l2": "inputs larger than L2 (sinogram 566 MB, volume 604 MB)",
                       "form": "batched: all slices per launch, one CUDA graph per iteration"},
            "cgls_iter_per_s": world * args.steps / t_cg, "gpu_launches": 2 * args.steps,
            "clocks": clk}
    line.update({k: d[k] for k in ("mlem_iter_per_s", "fp_ms", "bp_ms", "projector_rays_per_s",
                                   "plain_iter_per_s", "batched_over_plain", "roofline",
                                   "gather_roofline", "e2e", "cpu_baseline")})
    return line


# ------------------------------------------------------- other workloads
def ellipsoids(torch, dev, n, count, axes, seed):
    """ellipsoid_phantom on the device (see there)."""
    return torch.from_numpy(ellipsoid_phantom(n, count, axes, seed)).to(dev)


def line_common(args, workload, value, unit, t_step, cfg, **extra):
    d = {"metric": METRIC, "value": value, "unit": unit, "n_gpus": 1, "steps": args.steps,
         "warmup": args.warmup, "ms_per_step": 1000.0 * t_step, "higher_is_better": True,
         "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
         "config": dict({"workload": workload}, **cfg)}
    d.update(extra)
    return d


def uneven_problems(torch, dev, count=64):
    """64 seeded uneven parallel-beam problems (SeedSequence(4).spawn(64)):
    width w ~ U{64..384}, rows nz ~ U{8..64}, angles ~ U{90..900} over
    [0, pi), round(1.5 w) detector columns, lambda log-uniform in
    [1e-3, 1e-1]; 10 ellipses per slice projected on a w x w x nz grid,
    Gaussian noise of 2 % of the largest value.  Returns host pixel arrays
    (n_angles, n_v, n_h) with degrees and lambdas."""
    import numpy as np
    from ccpi.reconstruction.device import Plan
    out = []
    for ss in np.random.SeedSequence(4).spawn(count):
        rng = np.random.default_rng(ss)
        w = int(rng.integers(64, 385))
        nz = int(rng.integers(8, 65))
        na = int(rng.integers(90, 901))
        nh = int(round(1.5 * w))
        lam = float(np.exp(rng.uniform(np.log(1e-3), np.log(1e-1))))
        deg = np.linspace(0.0, 180.0, na, endpoint=False).astype(np.float32)
        c = torch.arange(w, device=dev, dtype=torch.float32) + 0.5 - w / 2
        X, Y = c.view(w, 1), c.view(1, w)
        vol = torch.zeros((w, w, nz), device=dev)
        for k in range(nz):
            sl = torch.zeros((w, w), device=dev)
            for _ in range(10):
                cx, cy = rng.uniform(-0.4, 0.4, 2) * w
                a, b = rng.uniform(0.04, 0.31, 2) * w
                th = rng.uniform(0, math.pi)
                d = rng.uniform(0.1, 1.0)
                xr = (X - cx) * math.cos(th) + (Y - cy) * math.sin(th)
                yr = -(X - cx) * math.sin(th) + (Y - cy) * math.cos(th)
                sl += ((xr / a) ** 2 + (yr / b) ** 2 <= 1.0).float() * d
            vol[:, :, k] = sl
        ang = math.pi * (deg.astype(np.float64) / 180.0)
        h = np.arange(nh) - (nh - 1) / 2.0
        v = np.arange(nz) - (nz - 1) / 2.0
        p = Plan("parallel", ang, h, v, (-w / 2, -w / 2, -nz / 2), (1.0, 1.0, 1.0), (w, w, nz))
        s = p.forward(vol).cpu().numpy()  # (na, nh, nz)
        p.close()
        s = s + rng.normal(0.0, 0.02 * np.abs(s).max(), s.shape).astype(np.float32)
        out.append(dict(pixels=np.ascontiguousarray(s.transpose(0, 2, 1), np.float32),
                        deg=deg, lam=lam))
    return out


def run_uneven(args):
    """64 uneven CGLS-Tikhonov and CGLS-TV problems, 40 iterations, one
    CUDA graph per iteration holding all 64 problems.  A step is one
    iteration of the whole batch."""
    import numpy as np
    import torch

    from ccpi.reconstruction.device import Session, pack_parallel, parallel_api_plan, solve_batched
    from ccpi.reconstruction.parallelbeam import alg as A
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    probs = uneven_problems(torch, dev)
    niter = 40
    plans, sinos = [], []
    for p in probs:
        na, nv, nh = p["pixels"].shape
        plan, nvp, voff = parallel_api_plan(na, nv, nh, p["deg"], 0.0, 1)
        plans.append(plan)
        sinos.append(pack_parallel(torch.from_numpy(p["pixels"]).to(dev), nvp, voff))
    # the autotuner picks each plan's projector launch shapes
    t0 = time.perf_counter()
    tuned = [pl.autotune() for pl in plans]
    t_tune = time.perf_counter() - t0
    vw_counts = {}
    for _, vw in tuned:
        vw_counts[str(vw)] = vw_counts.get(str(vw), 0) + 1
    lams = [p["lam"] for p in probs]
    V = sum(int(np.prod(pl.shape)) for pl in plans)
    P = sum(int(np.prod(pl.sino_shape)) for pl in plans)
    res = {}
    clocks = Clocks(0)
    for alg, name in ((3, "cgls_tikhonov"), (4, "cgls_TVreg")):
        xs = [torch.zeros(pl.shape, device=dev) for pl in plans]
        solve_batched(plans, alg, sinos, xs, 2, lams)  # warm-up (graph, caches)
        xs = [torch.zeros(pl.shape, device=dev) for pl in plans]
        t = cuda_time(torch, lambda: solve_batched(plans, alg, sinos, xs, niter, lams))
        # plain: problems one at a time, host-driven iterations, on a sample
        sample = list(range(0, len(plans), 8))
        tp = 0.0
        for i in sample:
            y = torch.zeros(plans[i].shape, device=dev)
            tp += cuda_time(torch, lambda: plans[i].solve(alg, sinos[i], y, niter, lams[i],
                                                         plain=True))
        t_plain = tp * len(plans) / len(sample)
        # the kernels alone: every problem's graph-captured iteration timed
        # on its own (data resident), summed over the 64 problems; no
        # batched form of the same kernels can beat this sum by more than
        # the overlap of problems too small to fill the GPU
        t_kern = 0.0
        for i, pl in enumerate(plans):
            y = torch.zeros(pl.shape, device=dev)
            sess = Session(pl, alg, sinos[i], y, 3, lams[i])
            sess.run(1)
            t_kern += cuda_time(torch, lambda: sess.run(2)) / 2.0
            sess.finish()
            sess.close()
        res[name] = {"batched_s": t, "plain_s": t_plain, "kernels_s": t_kern * niter}
    clk = clocks.stop()
    # e2e through the host-buffer batched call (Tikhonov)
    t0 = time.perf_counter()
    A.reconstruct_batched("cgls_tikhonov", [p["pixels"] for p in probs], [p["deg"] for p in probs],
                          0.0, 1, niter, 1, True, regularize=lams)
    t_e2e = time.perf_counter() - t0
    t_tik = res["cgls_tikhonov"]["batched_s"]
    peak, peak_kind = load_peaks()
    it_bytes = 4.0 * (12 * V + 4 * P)
    cpu = None if args.no_cpu else uneven_cpu_sample(probs)
    print(json.dumps(line_common(
        args, "64 uneven parallel-beam CGLS-Tikhonov and CGLS-TV problems (64^2x8 .. 384^2x64 "
              "volumes, 90-900 angles, 1.5x detector columns, 2% noise), 40 iterations, all 64 "
              "in one graph per iteration", niter / t_tik, "iter/s", t_tik / niter,
        {"problems": len(probs), "voxels": V, "pixels": P, "iterations": niter,
         "form": "batched: 64 problems per graph launch",
         "autotune": {"seconds": t_tune, "bp_slices_per_lane_chosen": vw_counts}},
        tv_iter_per_s=niter / res["cgls_TVreg"]["batched_s"],
        plain_iter_per_s={k: niter / v["plain_s"] for k, v in res.items()},
        kernels_only_iter_per_s={k: niter / v["kernels_s"] for k, v in res.items()},
        plain_over_kernels_only={k: v["plain_s"] / v["kernels_s"] for k, v in res.items()},
        batched_over_plain={k: v["plain_s"] / v["batched_s"] for k, v in res.items()},
        roofline={"bound": "hbm", "kernel": "one regularised CGLS iteration of the batch",
                  "achieved": it_bytes / (t_tik / niter) / 1e9, "peak": peak, "unit": "GB/s",
                  "frac": it_bytes / (t_tik / niter) / 1e9 / peak, "peak_kind": peak_kind,
                  "algorithmic_bytes_per_iteration": it_bytes, "traffic": None},
        e2e={"value": niter / t_e2e, "unit": "iter/s",
             "h2d_bytes_per_step": sum(p["pixels"].nbytes for p in probs) / niter,
             "d2h_bytes_per_step": 4.0 * V / niter,
             "call": "parallelbeam.alg.reconstruct_batched('cgls_tikhonov', 64 problems)"},
        clocks=clk, cpu_baseline=cpu)))


def uneven_cpu_sample(probs):
    """The reference's own cgls_tikhonov on the 4 smallest of the 64
    problems, t(2 iterations) - t(1), scaled to one iteration of all 64 by
    their share of n_angles x n_v x n_h^2 (the projectors' work)."""
    O = oracle()
    if not O.reference_available():
        return None
    threads = os.cpu_count() or 1
    work = lambda p: p["pixels"].shape[0] * p["pixels"].shape[1] * p["pixels"].shape[2] ** 2  # noqa
    sel = sorted(range(len(probs)), key=lambda i: work(probs[i]))[:4]
    t_sel = 0.0
    for i in sel:
        p = probs[i]
        times = []
        for it in (1, 2):
            t0 = time.perf_counter()
            with O.quiet():
                O.ref_pb_reconstruct(3, p["pixels"], p["deg"], 0.0, 1, it, True, lam=p["lam"],
                                     nthreads=threads)
            times.append(time.perf_counter() - t0)
        t_sel += max(times[1] - times[0], 1e-9)
    scale = sum(work(p) for p in probs) / sum(work(probs[i]) for i in sel)
    t_batch_iter = t_sel * scale
    return {"value": 1.0 / t_batch_iter, "unit": "iter/s", "cores": threads, "kind": "reference",
            "sample": "reference cgls_tikhonov on the 4 smallest problems (%s); t(2 iter) - "
                      "t(1 iter), scaled to all 64 by n_angles x n_v x n_h^2" % sel}


def run_autograd(args):
    """Differentiable cone projector: 8 volumes of 256^3 seeded ellipsoids
    (2 mm voxels), 360 angles over [0, 2 pi), 384 x 384 detector of 1.6 mm
    pixels, source/detector 500 mm; loss ||A x - y||^2 against noisy
    sinograms, minimised by Adam.  A step is one Adam step over the batch
    (8 forward and 8 back projections)."""
    import torch

    from ccpi.reconstruction.autograd import Projector
    from ccpi.reconstruction.device import cone_plan
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n, na, nd, nb = 256, 360, 384, 8
    plan = cone_plan(n, 2.0, na, nd, 1.6, 500.0, 500.0)
    bp_kernel, t_tune = pick_cone_bp(plan, args.cone_bp)
    A = Projector(plan)
    xt = torch.stack([ellipsoids(torch, dev, n, 40, (5.0, 60.0), seed=50 + b) for b in range(nb)])
    with torch.no_grad():
        y = A(xt)
        gen = torch.Generator(device=dev).manual_seed(5)
        y += 0.01 * float(y.abs().max()) * torch.randn(y.shape, device=dev, generator=gen)
    x = torch.zeros_like(xt, requires_grad=True)
    opt = torch.optim.Adam([x], lr=0.02)

    def step():
        opt.zero_grad()
        r = A(x) - y
        loss = (r * r).sum()
        loss.backward()
        opt.step()
        return loss
    l0 = float(step().detach())
    for _ in range(max(args.warmup - 1, 0)):
        step()
    clocks = Clocks(0)
    t = cuda_time(torch, step, args.steps)
    clk = clocks.stop()
    l1 = float(step().detach())
    # checks at full size on one volume: dot test
    with torch.no_grad():
        g = torch.Generator(device=dev).manual_seed(9)
        u = torch.rand((n, n, n), device=dev, generator=g)
        w = torch.rand(plan.sino_shape, device=dev, generator=g)
        lhs = float((plan.forward(u).double() * w.double()).sum())
        rhs = float((u.double() * plan.backward(w).double()).sum())
    P = na * nd * nd
    t_fp = cuda_time(torch, lambda: plan.forward(u), 2)
    t_bp = cuda_time(torch, lambda: plan.backward(w), 2)
    print(json.dumps(line_common(
        args, "differentiable cone projector: 8 x 256^3 ellipsoid volumes, 360 angles over "
              "2 pi, 384^2 detector at 1.6 mm, 2 mm voxels, source/detector 500 mm, Adam on "
              "||Ax - y||^2", 1.0 / t, "step/s", t,
        {"batch": nb, "grid": [n, n, n], "angles": na, "detector": [nd, nd]},
        fp_ms=1000 * t_fp, bp_ms=1000 * t_bp,
        projector_rays_per_s={"forward": P / t_fp, "backward": P / t_bp},
        loss_first=l0, loss_after=l1, dot_test_rel=abs(lhs - rhs) / abs(lhs),
        back_projector={"kernel": bp_kernel, "choice": args.cone_bp, "autotune_seconds": t_tune},
        # per step: one batched forward launch; the batched back projection
        # is one gather launch, or one scatter launch per volume
        gpu_launches=(1 + (nb if bp_kernel == "cb_bp_scatter" else 1)) * args.steps,
        clocks=clk)))


def run_cone_projectors(args):
    """The cone workload's projectors alone: one forward and one back
    projection per step on the 512^3 CGLS workload's geometry (or, with
    --cone-n 256, the 256^3 / 360-angle / 384^2 geometry), CUDA events on
    the launching stream.  Also the command that profiler captures of the
    cone kernels run."""
    import torch

    from ccpi.reconstruction.device import cone_plan
    dev = torch.device("cuda", 0)
    torch.cuda.set_device(dev)
    n, vs, na, nd, px = cone_geometry(args.cone_n)
    plan = cone_plan(n, vs, na, nd, px, CS2O, CO2D)
    bp_kernel, _ = pick_cone_bp(plan, args.cone_bp)
    vol = torch.from_numpy(ellipsoid_phantom(n, 40, (10.0 * n / CN, 120.0 * n / CN), seed=3)).to(dev)
    sino = plan.forward(vol)
    out = torch.empty_like(vol)
    for _ in range(args.warmup):
        plan.forward(vol, sino)
        plan.backward(sino, out)
    t_fp = cuda_time(torch, lambda: plan.forward(vol, sino), args.steps)
    t_bp = cuda_time(torch, lambda: plan.backward(sino, out), args.steps)
    V, P = n ** 3, na * nd * nd
    peak, peak_kind = load_peaks()
    print(json.dumps(line_common(
        args, f"cone-beam projectors, {n}^3 ellipsoid phantom, {na} angles, {nd}^2 detector",
        P / t_bp, "rays/s", t_fp + t_bp, {"grid": [n] * 3, "angles": na, "detector": [nd, nd]},
        fp_ms=1000 * t_fp, bp_ms=1000 * t_bp,
        projector_rays_per_s={"forward": P / t_fp, "backward": P / t_bp},
        roofline={"bound": "hbm", "kernel": bp_kernel, "achieved": 4.0 * (V + P) / t_bp / 1e9,
                  "peak": peak, "unit": "GB/s", "frac": 4.0 * (V + P) / t_bp / 1e9 / peak,
                  "peak_kind": peak_kind},
        gpu_launches=2 * args.steps)))
    plan.close()


# -------------------------------------------------------------------- main
def main():
    args = parse()
    if args.impl == "reference":
        return run_reference(args)
    if args.workload in ("uneven", "autograd", "cone-projectors"):
        return {"uneven": run_uneven, "autograd": run_autograd,
                "cone-projectors": run_cone_projectors}[args.workload](args)
    import torch
    import torch.distributed as dist

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

    if args.workload == "sirt":
        line = sirt_part(args, torch, dev, world, rank, barrier, max_over_ranks, full_line=True)
    else:
        line = cone_line(args, torch, dev, world, rank, barrier, max_over_ranks)
        if not args.no_parallel:
            line["parallel_sirt"] = sirt_part(args, torch, dev, world, rank, barrier,
                                              max_over_ranks)
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the cube Coulomb operator at 481^3 (the headline workload).

Workload: 481^3 grid (80 cells x 6 + 1 per axis, step 0.1 bohr, box
[-24, 24]^3), density = 32 seeded Gaussians (alpha log-uniform in [0.1, 20],
q ~ U[0.5, 2], centres ~ U[-10, 10]^3), 64 t-points (32 Gauss-Legendre on
[0, 2] + 32 log-mapped on [2, 1e3]).  One step = one application of the
operator V = sum_p w_p (Tx (x) Ty (x) Tz)_p rho + coda rho to the resident
density, energy integral included.  Metric: grid points per second (Mpts/s).

Default run: the split-precision tensor-core operator in its fp16x3 mode
(two FP16 parts per operand with power-of-two stage scales, three products,
the tensor core's toward-zero rounding bias removed; within 1e-6 relative
potential error and 1e-7 relative energy error of the FP64 operator on
every configuration tested) with the FP64 GPU operator timed beside it and
the error of the former against the latter reported; the bf16x3 (two BF16
parts: meets the bounds here but not on the 121^3 configuration) and
bf16x6 (three BF16 parts, six products) modes are timed and checked the same
way and reported under "alternatives".  `--precision fp64` benchmarks the
drop-in alone.
`--impl reference` times the CPU restatement of the reference algorithm
(oracle/, DGEMM per mode product) on the host cores instead.

Multi-GPU: the operator does not shard in this build; N ranks run N
independent replicas ("scaling": "weak"), timed as the max over ranks.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_CELL = 80
STEP = 0.1
NLIN = NLOG = 32
TLIN, TLOG = 2.0, 1.0e3
SEED = 3
N_GAUSS = 32
METRIC = "Coulomb-op Mpts/s @481^3: mixed vs FP64 on B200 at <=1e-6 rel err; CPU ref shown"


def gaussians(seed=SEED, ng=N_GAUSS):
    rng = np.random.default_rng(seed)
    q = rng.uniform(0.5, 2.0, ng)
    a = np.exp(rng.uniform(np.log(0.1), np.log(20.0), ng))
    c = rng.uniform(-10.0, 10.0, (ng, 3))
    return q, a, c


def axis_points(n_cell=N_CELL, step=STEP):
    qmin = -0.5 * n_cell * 6 * step
    return qmin + step * np.arange(n_cell * 6 + 1)


def density_torch(pts, q, a, c, device):
    """rho(x,y,z) on the device as a flat float64 tensor, x fastest."""
    import torch

    x = torch.tensor(pts, dtype=torch.float64, device=device)
    n = len(pts)
    rho = torch.zeros((n, n, n), dtype=torch.float64, device=device)  # [z, y, x]
    for qi, ai, ci in zip(q, a, c):
        norm = qi * (ai / np.pi) ** 1.5
        ex = torch.exp(-ai * (x - ci[0]) ** 2)
        ey = torch.exp(-ai * (x - ci[1]) ** 2)
        ez = torch.exp(-ai * (x - ci[2]) ** 2)
        rho += norm * ez[:, None, None] * ey[None, :, None] * ex[None, None, :]
    return rho.reshape(-1)


class ClockSampler:
    """nvidia-smi clock/throttle sampling during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index: int):
        self.index = index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.Q}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except FileNotFoundError:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                smax.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["no samples"]}
        load = [s for s in sm if s > 0.5 * max(sm)]
        return {"sm_mhz": float(np.median(load or sm)), "sm_max_mhz": float(max(smax)),
                "reasons": sorted(reasons), "samples": len(sm)}


def dist_setup():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        import datetime

        import torch
        import torch.distributed as dist

        backend = "nccl" if torch.cuda.is_available() else "gloo"  # gloo: CPU tests
        if backend == "nccl":
            torch.cuda.set_device(local)
        dist.init_process_group(backend, timeout=datetime.timedelta(seconds=600))
    return world, rank, local


def barrier_max(value: float, world: int) -> float:
    if world == 1:
        return value
    import torch
    import torch.distributed as dist

    dev = "cuda" if dist.get_backend() == "nccl" else "cpu"
    t = torch.tensor([value], dtype=torch.float64, device=dev)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def barrier(world: int):
    if world > 1:
        import torch.distributed as dist

        dist.barrier()


def peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(path):
        with open(path) as f:
            d = json.load(f)
        return d, "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0, "bf16_tflops_sustained": 1400.0}, "fallback"


def profiled_traffic(kernel: str, workload: str, precision: str | None = None):
    """Per-launch DRAM bytes of a kernel from the committed ncu summary."""
    path = os.path.join(ROOT, "profiles", "roofline_traffic.txt")
    if not os.path.exists(path):
        return None
    for ln in open(path):
        kv = dict(x.split("=", 1) for x in ln.split() if "=" in x)
        if (kv.get("kernel") == kernel and kv.get("workload") == workload
                and (precision is None or kv.get("precision", precision) == precision)):
            try:
                return float(kv["traffic_bytes_per_launch"])
            except (KeyError, ValueError):
                return None
    return None


def headline_config(n: int, world: int) -> dict:
    """The `config` of the headline line, shared by the GPU and CPU arms."""
    return {"workload": f"coulomb_cube_{n}", "points_per_axis": n, "step_bohr": STEP,
            "t_points": NLIN + NLOG, "gaussians": N_GAUSS, "seed": SEED,
            "l2": f"inputs larger than L2 (rho {8 * n ** 3 / 1e9:.2f} GB)",
            "parallelism": f"replicas x{world}"}


# ---------------------------------------------------------------------------
# CPU arms
# ---------------------------------------------------------------------------
_CPU_SETUP = {}


def _cpu_setup(n_cell, step):
    key = (n_cell, step)
    if key not in _CPU_SETUP:
        from oracle import oracle as O

        qmin = -0.5 * n_cell * 6 * step
        g = O.Grid3D.cube(qmin, n_cell, step)
        q, a, c = gaussians()
        rho = O.gauss_cube(g, q, a, c)
        tp, tw = O.gauss_quad(NLIN, NLOG, 0.0, TLIN, TLOG)
        T = O.coulomb_matrix(g.axes[0], g.axes[0].points, tp)
        w = O.coulomb_weights(tw)
        _CPU_SETUP.clear()
        _CPU_SETUP[key] = (g, rho, tp, T, w)
    return _CPU_SETUP[key]


def cpu_sample(n_cell=N_CELL, step=STEP, ip=0):
    """Times the CPU restatement (oracle, numpy/OpenBLAS DGEMM per mode
    product, all host threads) on one t-point (index ip) of the 481^3
    operator: 1/64 of an apply.  Returns (seconds, points, t-points)."""
    from oracle import oracle as O

    g, rho, tp, T, w = _cpu_setup(n_cell, step)
    ip = ip % len(tp)
    t0 = time.perf_counter()
    O.transform_cube_blas(T, T, T, w, rho, 0.0, p_subset=[ip])
    return time.perf_counter() - t0, float(g.shape[0]) ** 3, len(tp)


def run_reference(args, world, rank):
    """The reference algorithm's CPU path on the host cores.  One step = one
    t-point of the 481^3 apply (1/64 of the work of one apply; the dense
    DGEMMs cost the same for every t-point), cycling through the t-points;
    the line's rate is points x t-points processed / time, i.e. the apply
    rate, and the per-apply time it implies is reported as extrapolated."""
    if rank != 0:
        return
    times = []
    npts = n_t = None
    for i in range(args.warmup + args.steps):
        dt, npts, n_t = cpu_sample(ip=i * 13)
        if i >= args.warmup:
            times.append(dt)
    sample_s = float(np.mean(times))
    value = npts / (sample_s * n_t) / 1e6
    n = N_CELL * 6 + 1
    cores = os.cpu_count()
    sample = (f"{args.steps} timed steps of one t-point each (of {n_t}) of the {n}^3 apply, "
              f"OpenBLAS DGEMM on {cores} host threads")
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "Mpts/s",
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": sample_s * 1e3, "step": f"one t-point of {n_t} (1/{n_t} of an apply)",
        "extrapolated_ms_per_apply": sample_s * n_t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": headline_config(n, world),
        "cpu_baseline": {"value": value, "unit": "Mpts/s", "cores": cores, "kind": "port",
                         "sample": sample},
        "e2e": {"value": value, "unit": "Mpts/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# GPU arm
# ---------------------------------------------------------------------------
def run_e2e(op, rho, n, npts, world, args):
    """The same metric through the public API with pinned HOST buffers: every
    step copies rho in and V (and the energy) back inside the timed region.
    Headline: the batched host-pointer call (dage_op3d_apply_batched), whose
    pipeline overlaps each step's copies with the neighbouring steps'
    compute; beside it the one-apply-per-call form, copies and compute in
    series."""
    import torch

    import dage_b200 as dage

    def pinned():
        return torch.empty(rho.numel(), dtype=torch.float64, pin_memory=True)

    rho_h, V_h, V2_h = pinned(), pinned(), pinned()
    rho_h.copy_(rho.cpu())
    fview = lambda t: t.numpy().reshape(n, n, n).T  # Fortran-ordered (x, y, z) view
    rho_np, V_np, V2_np = fview(rho_h), fview(V_h), fview(V2_h)
    e2e_steps = max(2, min(2 * args.steps, 16))
    # sequential: one dage_op3d_apply per step
    op.apply(rho_np, out=V_np, energy=True)
    barrier(world)
    t0 = time.perf_counter()
    for _ in range(e2e_steps):
        op.apply(rho_np, out=V_np, energy=True)
    seq_s = barrier_max((time.perf_counter() - t0) / e2e_steps, world)
    # pipelined: all steps in one batched call, outputs alternating between
    # two pinned buffers
    outs = [V_np if i % 2 == 0 else V2_np for i in range(e2e_steps)]
    dage.apply_batched([op] * 2, [rho_np] * 2, outs[:2], energy=True)  # staging slots
    barrier(world)
    t0 = time.perf_counter()
    dage.apply_batched([op] * e2e_steps, [rho_np] * e2e_steps, outs, energy=True)
    e2e_s = barrier_max((time.perf_counter() - t0) / e2e_steps, world)
    return {"value": world * npts / e2e_s / 1e6, "unit": "Mpts/s",
            "h2d_bytes_per_step": int(8 * npts), "d2h_bytes_per_step": int(8 * npts + 8),
            "ms_per_step": e2e_s * 1e3, "steps": e2e_steps,
            "api": "dage_op3d_apply_batched, host pointers (copies overlapped with compute)",
            "sequential": {"value": world * npts / seq_s / 1e6, "ms_per_step": seq_s * 1e3,
                           "api": "dage_op3d_apply per step, host pointers"}}


def band_fraction(T, bk=64, bn=128):
    """Fraction of the dense K range that the stage kernels issue work for:
    per t-point and 128-row tile of T (i_out, j_in, p), the K blocks of bk
    between the first and last entry above 2^-64 of its row's power-of-two
    scale (the kernels' band rule; identical for the three axes of a cube)."""
    no, ni, P = T.shape
    nkb = -(-ni // bk)
    last = ni - (nkb - 1) * bk
    issued = 0.0
    for p in range(P):
        A = np.abs(T[:, :, p])
        s = np.exp2(np.ceil(np.log2(np.maximum(A.max(axis=1), 1e-300))))
        big = A > np.ldexp(s, -64)[:, None]
        for t0 in range(0, no, bn):
            cols = np.nonzero(big[t0:t0 + bn].any(axis=0))[0]
            lo, hi = (cols[0] // bk, cols[-1] // bk) if cols.size else (0, 0)
            k = (hi - lo) * bk + (last if hi == nkb - 1 else bk)
            issued += min(bn, no - t0) * k
    return issued / (no * ni * P)


def analytic_errors(V, V64, ncell, q, a, c, dev):
    """Max and RMS error, relative to max |Va| and RMS Va, of the operator's
    potentials against the analytic sum q erf(sqrt(a) r)/r of the Gaussians,
    at the grid points (z slabs of 32 planes)."""
    import torch

    x = torch.tensor(axis_points(ncell), dtype=torch.float64, device=dev)
    n = len(x)
    out = {}
    vmax = 0.0
    ssq = 0.0
    err = {"mixed": [0.0, 0.0], "fp64": [0.0, 0.0]}
    for z0 in range(0, n, 32):
        zs = x[z0:z0 + 32]
        Z, Y, X = torch.meshgrid(zs, x, x, indexing="ij")
        Va = torch.zeros_like(X)
        for qi, ai, ci in zip(q, a, c):
            r = torch.sqrt((X - ci[0]) ** 2 + (Y - ci[1]) ** 2 + (Z - ci[2]) ** 2)
            small = r < 1e-12
            val = qi * torch.erf(np.sqrt(ai) * r) / torch.where(small, torch.ones_like(r), r)
            Va += torch.where(small, torch.full_like(r, qi * 2 * np.sqrt(ai / np.pi)), val)
        sl = slice(z0 * n * n, (z0 + len(zs)) * n * n)
        vmax = max(vmax, float(Va.abs().max()))
        ssq += float((Va * Va).sum())
        for key, W in (("mixed", V), ("fp64", V64)):
            dv = W[sl].reshape(Va.shape) - Va
            err[key][0] = max(err[key][0], float(dv.abs().max()))
            err[key][1] += float((dv * dv).sum())
    for key in err:
        out[key] = {"max_rel": err[key][0] / vmax, "rms_rel": float(np.sqrt(err[key][1] / ssq))}
    out["vs"] = "analytic sum q erf(sqrt(a) r)/r at the grid points"
    return out


def run_gpu(args, world, rank, local):
    import torch

    import dage_b200 as dage
    from dage_b200 import build as b

    b.build()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    ncell = args.n_cell
    n = ncell * 6 + 1
    npts = float(n) ** 3
    g = dage.Grid3D.cube(-0.5 * ncell * 6 * STEP, ncell, STEP)
    quad = dage.GaussQuad(NLIN, NLOG, 0.0, TLIN, TLOG)
    q, a, c = gaussians()
    rho = density_torch(axis_points(ncell), q, a, c, dev)
    prec = args.precision
    op = dage.Coulomb3D(g, quad=quad, precision=prec)
    V = torch.empty_like(rho)

    # -- device-resident timed region ---------------------------------------
    for _ in range(args.warmup):
        op.apply(rho, out=V, energy=True)
    op.set_timing(True)
    clk = ClockSampler(local)
    barrier(world)
    torch.cuda.synchronize()
    clk.start()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record()
    energy = None
    for _ in range(args.steps):
        _, energy = op.apply(rho, out=V, energy=True)
    e1.record()
    torch.cuda.synchronize()
    clocks = clk.stop()
    barrier(world)
    ms = e0.elapsed_time(e1) / args.steps
    ms = barrier_max(ms, world)
    value = world * npts / (ms / 1e3) / 1e6
    launches = sum(op.timing(k)[0] for k in range(3))
    k_launches, k_ms = op.timing(0)
    op.set_timing(False)

    # -- dominant kernel roofline -------------------------------------------
    pk, src = peaks()
    nprod = {"fp64": 1, "bf16x3": 3, "bf16x6": 6, "fp16x3": 3}[prec]
    # one stage of one t-point: M = n^2, N = K = n; the last stage's launches
    # cover up to 8 t-points, so rates use the total stage time of an apply
    dense_flops = 2.0 * n ** 4 * nprod
    band = band_fraction(op.matrix(0), bk=16 if prec == "fp64" else 32)
    stage_flops = dense_flops * band    # work the banded contraction issues
    stage_s = k_ms / args.steps / 1e3   # contraction kernels' time per apply
    apply_flops = 3 * (NLIN + NLOG) * stage_flops
    achieved = apply_flops / stage_s / 1e12
    avg_launch_s = k_ms / max(k_launches, 1) / 1e3
    if prec == "fp64":
        peak, peak_src = 40.0, "nominal B200 FP64 (no measured FP64 peak)"
        kname = "stage_fp64_kernel"
    else:
        peak, peak_src = pk["bf16_tflops_sustained"], f"{src} bf16_tflops_sustained"
        kname = "stage_bf16_kernel"
    traffic = profiled_traffic(kname, f"coulomb_cube_{n}", None if prec == "fp64" else prec)
    roof = {"bound": "tensor", "achieved": achieved, "peak": peak, "unit": "TFLOP/s",
            "frac": achieved / peak, "traffic": traffic, "kernel": kname,
            "peak_source": peak_src,
            "flops_per_launch": apply_flops * args.steps / max(k_launches, 1),
            "flops_per_stage_and_tpoint": stage_flops, "band_fraction": band,
            "dense_equiv_tflops": achieved / band,
            "avg_launch_ms": avg_launch_s * 1e3, "launches_timed": k_launches,
            "stage_ms_per_apply": stage_s * 1e3}

    # -- accuracy against the FP64 GPU operator and the analytic potential --
    accuracy = None
    alternative = None
    fp64_mpts = None
    build_ms = None
    if prec != "fp64" and not args.skip_fp64:
        torch.cuda.synchronize()
        tb = time.perf_counter()
        op64 = dage.Coulomb3D(g, quad=quad, precision="fp64")  # T_p matrices built on the GPU
        torch.cuda.synchronize()
        build_ms = (time.perf_counter() - tb) * 1e3
        V64 = torch.empty_like(rho)
        _, E64 = op64.apply(rho, out=V64, energy=True)
        torch.cuda.synchronize()
        f0 = torch.cuda.Event(enable_timing=True)
        f1 = torch.cuda.Event(enable_timing=True)
        nrep = max(1, args.fp64_steps)
        clk64 = ClockSampler(local)
        clk64.start()
        f0.record()
        for _ in range(nrep):
            op64.apply(rho, out=V64, energy=True)
        f1.record()
        torch.cuda.synchronize()
        clocks64 = clk64.stop()
        fp64_ms = f0.elapsed_time(f1) / nrep
        fp64_mpts = npts / (fp64_ms / 1e3) / 1e6
        d = (V - V64).abs()
        accuracy = {
            "vs": "fp64 GPU operator",
            "max_rel": float(d.max() / V64.abs().max()),
            "rms_rel": float(torch.sqrt((d * d).mean() / (V64 * V64).mean())),
            "energy_rel": abs(energy - E64) / abs(E64),
            "fp64_ms_per_step": fp64_ms,
            "fp64_mpts": fp64_mpts,
            "speedup_vs_fp64": fp64_ms / ms,
            "fp64_steps": nrep, "fp64_clocks": clocks64,
            "vs_analytic": analytic_errors(V, V64, ncell, q, a, c, dev),
        }
        if clocks.get("sm_mhz") and clocks64.get("sm_mhz"):
            # the same ratio in cycles (time x median SM clock of each arm)
            accuracy["speedup_vs_fp64_cycles"] = (fp64_ms * clocks64["sm_mhz"]) / (ms * clocks["sm_mhz"])
        del op64
        if not args.skip_alt:
            # the other split-precision modes on the same input, same checks
            alternative = []
            for other in ("fp16x3", "bf16x3", "bf16x6"):
                if other == prec:
                    continue
                opa = dage.Coulomb3D(g, quad=quad, precision=other)
                Va = torch.empty_like(rho)
                for _ in range(args.warmup):
                    opa.apply(rho, out=Va, energy=True)
                torch.cuda.synchronize()
                a0 = torch.cuda.Event(enable_timing=True)
                a1 = torch.cuda.Event(enable_timing=True)
                a0.record()
                for _ in range(args.steps):
                    _, Ea = opa.apply(rho, out=Va, energy=True)
                a1.record()
                torch.cuda.synchronize()
                a_ms = a0.elapsed_time(a1) / args.steps
                da = (Va - V64).abs()
                alternative.append({
                    "precision": other, "ms_per_step": a_ms, "value": npts / (a_ms / 1e3) / 1e6,
                    "unit": "Mpts/s", "speedup_vs_fp64": fp64_ms / a_ms,
                    "max_rel": float(da.max() / V64.abs().max()),
                    "rms_rel": float(torch.sqrt((da * da).mean() / (V64 * V64).mean())),
                    "energy_rel": abs(Ea - E64) / abs(E64),
                })
                del opa, Va
        del V64

    # -- end to end through the public API with host buffers -----------------
    e2e = None
    if not args.skip_e2e:
        e2e = run_e2e(op, rho, n, npts, world, args)

    cpu = None
    if rank == 0 and world == 1 and not args.skip_cpu:
        dts = [cpu_sample(n_cell=ncell, ip=13 * i)[0] for i in range(4)]
        dt = float(np.mean(dts[1:]))
        cores = os.cpu_count()
        cpu = {"value": npts / (dt * (NLIN + NLOG)) / 1e6, "unit": "Mpts/s", "cores": cores,
               "kind": "port",
               "sample": f"3 of the {NLIN + NLOG} t-points of the {n}^3 apply after one warm-up "
                         f"(OpenBLAS DGEMM, {cores} host threads); rate = points x t-points / time",
               "seconds_per_t_point": dt}

    if rank == 0:
        line = {
            "metric": METRIC, "value": value, "unit": "Mpts/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None,
            "dtype": {"fp64": "f64", "fp16x3": "f16"}.get(prec, "bf16"), "precision": prec,
            "data": "synthetic",
            "config": headline_config(n, world),
            "e2e": e2e, "roofline": roof, "cpu_baseline": cpu, "clocks": clocks,
            "gpu_launches": int(launches), "accuracy": accuracy, "energy": energy,
            "alternatives": alternative,
            "operator_build_ms": build_ms,
            "schedule": ({"ring_stages": op.schedule[0], "tpoint_group": op.schedule[1]}
                         if op.schedule else {"tiles": list(op.tiles)}),
        }
        print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# The other configurations of the path (not the headline line): each prints
# one JSON line of its own (bench.py --workload NAME)
# ---------------------------------------------------------------------------
def _timed(fn, steps, warmup, sync):
    import torch

    for _ in range(warmup):
        fn()
    sync()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record()
    for _ in range(steps):
        fn()
    e1.record()
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / steps


def _line(args, world, metric, value, unit, ms, dtype, config, clocks, launches, extra):
    line = {"metric": metric, "value": value, "unit": unit, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": dtype, "data": "synthetic",
            "config": config, "e2e": None, "roofline": None, "cpu_baseline": None,
            "clocks": clocks, "gpu_launches": launches}
    line.update(extra)
    print(json.dumps(line), flush=True)


def _gauss_cube(dev, n_cell, step, q, a, c):
    return density_torch(axis_points(n_cell, step), q, a, c, dev)


def _molecule_bubbles(dage, rng, nsets=1):
    """20 atoms uniform in a 30 bohr box, each a radial LIP grid of 199 points
    (33 cells, cell ends log-spaced on [1e-5, 15] bohr) with lmax 2 radial
    functions c r^l e^(-zeta r), c ~ U[-1, 1], zeta ~ U[0.5, 3]; and the
    301^3 cube (step 0.1) they are injected into.  nsets > 1: that many
    bubble sets (orbitals) on the same atoms, returned as a list."""
    gcube = dage.Grid3D.cube(-15.0, 50, 0.1)
    edges = np.concatenate([[0.0], 1e-5 * (15.0 / 1e-5) ** (np.arange(33) / 32)])
    rad = dage.Grid1D(0.0, 33, 7, 1, np.diff(edges) / 6)
    r = rad.coordinates()
    centers = rng.uniform(-15, 15, (20, 3))
    sets = []
    for _ in range(nsets):
        f = []
        for _ in range(20):
            fa = np.zeros((9, len(r)))
            for l in range(3):
                for m in range(-l, l + 1):
                    fa[l * (l + 1) + m] = (rng.uniform(-1, 1) * r ** l
                                           * np.exp(-rng.uniform(0.5, 3) * r))
            f.append(fa)
        sets.append(dage.Bubbles(centers, [rad] * 20, f, 2))
    return (sets[0] if nsets == 1 else sets), gcube


def run_workload(args, world, rank, local):
    import torch

    import dage_b200 as dage
    from dage_b200 import build as b

    b.build()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    sync = torch.cuda.synchronize
    clk = ClockSampler(local)
    wl = args.workload
    if wl == "coulomb_cube_121":
        # FP64 single box, 121^3 (20 cells, step 0.2), 2 Gaussians, 40 t-points
        rng = np.random.default_rng(SEED)
        q, a, c = rng.uniform(0.5, 2, 2), rng.uniform(0.5, 4, 2), rng.uniform(-3, 3, (2, 3))
        g = dage.Grid3D.cube(-12.0, 20, 0.2)
        rho = _gauss_cube(dev, 20, 0.2, q, a, c)
        op = dage.Coulomb3D(g, quad=dage.GaussQuad(20, 20, 0.0, TLIN, TLOG))
        V = torch.empty_like(rho)
        clk.start()
        ms = _timed(lambda: op.apply(rho, out=V, energy=True), args.steps, args.warmup, sync)
        clocks = clk.stop()
        # analytic potential sum q erf(sqrt(a) r) / r at the grid points
        x = torch.tensor(axis_points(20, 0.2), dtype=torch.float64, device=dev)
        Z, Y, X = torch.meshgrid(x, x, x, indexing="ij")
        Va = torch.zeros_like(X)
        for qi, ai, ci in zip(q, a, c):
            r = torch.sqrt((X - ci[0]) ** 2 + (Y - ci[1]) ** 2 + (Z - ci[2]) ** 2).clamp_min(1e-300)
            Va += qi * torch.erf(np.sqrt(ai) * r) / r
        err = float((V - Va.reshape(-1)).abs().max() / Va.abs().max())
        n = 121 ** 3
        _line(args, world, "Coulomb-op Mpts/s @121^3 FP64", n / ms / 1e3, "Mpts/s", ms, "f64",
              {"workload": wl, "points_per_axis": 121, "step_bohr": 0.2, "t_points": 40,
               "gaussians": 2, "seed": SEED}, clocks, 3 * 40 + 2,
              {"accuracy": {"vs": "analytic sum q erf(sqrt(a) r)/r", "max_rel": err}})
    elif wl in ("gbfmm_241", "gbfmm_241_adaptive", "helmholtz_gbfmm_241", "helmholtz_gbfmm_241"):
        # GBFMM, 241^3 (40 cells, step 0.2), 4^3 boxes, lmax 12, 16 Gaussians
        # (the adaptive variant: the reference's adaptive mode, level-1 moments;
        # the Helmholtz variant: kernel e^(-kappa r)/r at E = -0.5, kappa = 1).
        # --precision fp64 times the FP64 operator; any split mode times the
        # fp16x3 near field (the GBFMM's mixed form) beside the FP64 operator.
        adaptive = wl.endswith("adaptive")
        helm = wl.startswith("helmholtz")
        prec = "fp64" if args.precision == "fp64" else "fp16x3"
        rng = np.random.default_rng(SEED)
        q, a = rng.uniform(-1, 2, 16), rng.uniform(0.3, 6, 16)
        c = rng.uniform(-24, 24, (16, 3))
        g = dage.Grid3D.cube(-24.0, 40, 0.2)
        rho = _gauss_cube(dev, 40, 0.2, q, a, c)
        quad = dage.GaussQuad(20, 20, 0.0, TLIN, TLOG)

        def make(pr):
            return (dage.GBFMMHelmholtz3D(g, -0.5, lmax=12, quad=quad, precision=pr) if helm
                    else dage.GBFMMCoulomb3D(g, lmax=12, quad=quad, adaptive_mode=adaptive,
                                             precision=pr))
        op = make(prec)
        V = torch.empty_like(rho)
        clk.start()
        ms = _timed(lambda: op.apply(rho, out=V, energy=True), args.steps, args.warmup, sync)
        clocks = clk.stop()
        _, E = op.apply(rho, out=V, energy=True)
        extra = {}
        V64, E64 = V, E
        if prec != "fp64" and not args.skip_fp64:
            op64 = make("fp64")
            V64 = torch.empty_like(rho)
            ms64 = _timed(lambda: op64.apply(rho, out=V64, energy=True), max(2, args.steps // 3),
                          1, sync)
            _, E64 = op64.apply(rho, out=V64, energy=True)
            d = (V - V64).abs()
            s64 = V64.abs().max()
            extra["mixed_vs_fp64"] = {"max_rel": float(d.max() / s64),
                                      "rms_rel": float(d.pow(2).mean().sqrt() / s64),
                                      "energy_rel": abs(E - E64) / abs(E64),
                                      "fp64_ms_per_step": ms64,
                                      "speedup_vs_fp64": ms64 / ms}
            del op64
        n = 241 ** 3
        if not args.skip_fp64:
            Vd = torch.empty_like(rho)
            direct = dage.Coulomb3D(g, quad=quad)
            if helm:
                direct = dage.Helmholtz3D(direct, -0.5)
            _, Ed = direct.apply(rho, out=Vd, energy=True, coda=False)
            err = float((V64 - Vd).abs().max() / Vd.abs().max())
            extra["accuracy"] = {"vs": "single-box FP64 operator of the same kernel (no coda)",
                                 "fp64_gbfmm_max_rel": err,
                                 "fp64_gbfmm_energy_rel": abs(E64 - Ed) / abs(Ed)}
        _line(args, world, "GBFMM %s Mpts/s @241^3 %s (lmax 12, 4^3 boxes%s)"
              % ("Helmholtz (kappa 1)" if helm else "Coulomb",
                 "FP64" if prec == "fp64" else "fp16x3 near field",
                 ", adaptive mode" if adaptive else ""), n / ms / 1e3,
              "Mpts/s", ms, "f64" if prec == "fp64" else "f16",
              {"workload": wl, "points_per_axis": 241, "step_bohr": 0.2, "t_points": 40,
               "lmax": 12, "boxes": 64, "gaussians": 16, "seed": SEED, "precision": prec,
               "near_field_tiles": list(op.tiles)}, clocks, 3 * 40 + 9, extra)
    elif wl == "bubbles_inject_301":
        rng = np.random.default_rng(SEED)
        bub, gcube = _molecule_bubbles(dage, rng)
        cube = torch.zeros(301 ** 3, dtype=torch.float64, device=dev)
        clk.start()
        ms = _timed(lambda: bub.inject(gcube, cube=cube), args.steps, args.warmup, sync)
        clocks = clk.stop()
        n = 301 ** 3
        _line(args, world, "Bubbles->cube injection Mpts/s @301^3 (20 atoms, lmax 2)",
              n / ms / 1e3, "Mpts/s", ms, "f64",
              {"workload": wl, "points_per_axis": 301, "step_bohr": 0.1, "atoms": 20,
               "lmax": 2, "radial_points": 199, "seed": SEED}, clocks, 1,
              {"hbm_GBps": 16.0 * n / ms / 1e6})
    elif wl == "density_product_301":
        # Function3D_multiply of two orbitals (cube + lmax 2 bubbles each, 20
        # atoms) at 301^3: out = (c1 + B1)(c2 + B2) - B1*B2, B1*B2 lmax 4
        rng = np.random.default_rng(SEED)
        (b1, b2), gcube = _molecule_bubbles(dage, rng, nsets=2)
        br = b1 * b2
        n = 301 ** 3
        gen = torch.Generator(device=dev).manual_seed(SEED)
        c1 = torch.randn(n, dtype=torch.float64, device=dev, generator=gen)
        c2 = torch.randn(n, dtype=torch.float64, device=dev, generator=gen)
        out = torch.empty_like(c1)
        clk.start()
        ms = _timed(lambda: dage.multiply(gcube, c1, c2, b1, b2, br, out=out), args.steps,
                    args.warmup, sync)
        clocks = clk.stop()
        # the same product as separate passes (the reference GPU path's
        # structure: inject B1, inject B2, multiply, de-inject B1*B2)
        t1, t2 = torch.empty_like(c1), torch.empty_like(c2)

        def unfused():
            t1.copy_(c1)
            t2.copy_(c2)
            b1.inject(gcube, cube=t1)
            b2.inject(gcube, cube=t2)
            torch.mul(t1, t2, out=t1)
            br.inject(gcube, cube=t1, factor=-1.0)

        ms_unfused = _timed(unfused, max(1, args.steps // 2), 1, sync)
        err = float((t1 - out).abs().max() / out.abs().max())
        # the cusp form of the same product (Function3D_multiply_bubbles with
        # Taylor series, order 2): contaminants of both factors (other atoms'
        # bubbles and the cube), Taylor bubbles, their product, then the cube
        # product with those result bubbles
        def taylor_setup():
            ta = b1.taylor_series(gcube, c1, 2)
            tb = b2.taylor_series(gcube, c2, 2)
            return b1.multiply_taylor(b2, ta, tb)

        brt = taylor_setup()
        sync()
        reps = max(1, args.steps // 2)
        t0 = time.perf_counter()
        for _ in range(reps):
            brt = taylor_setup()
        sync()
        setup_ms = (time.perf_counter() - t0) * 1e3 / reps
        ms_cusp = _timed(lambda: dage.multiply(gcube, c1, c2, b1, b2, brt, out=t2),
                         max(1, args.steps // 2), 1, sync)
        _line(args, world, "Function3D product Mpts/s @301^3 (20 atoms, bubbles lmax 2 x 2 -> 4)",
              n / ms / 1e3, "Mpts/s", ms, "f64",
              {"workload": wl, "points_per_axis": 301, "step_bohr": 0.1, "atoms": 20,
               "lmax": [2, 2, 4], "radial_points": 199, "seed": SEED}, clocks, 1,
              {"hbm_GBps": 24.0 * n / ms / 1e6,
               "separate_passes": {"ms": ms_unfused, "launches": 4, "max_rel_diff": err},
               "taylor_cusp": {"setup_ms": setup_ms, "product_ms": ms_cusp, "taylor_order": 2,
                               "setup": "contaminants (bubbles + cube) and Taylor bubbles of "
                                        "both factors, option-(1) bubble product; host calls"}})
    elif wl in ("gbfmm_batch_256", "helmholtz_step_301"):
        rng = np.random.default_rng(SEED)
        if wl == "gbfmm_batch_256":
            nd, lmax = 256, 12
            cells = rng.choice([10, 15, 20, 25, 30], nd)
            energies = None
        else:
            nd, lmax = 64, 10
            cells = np.full(nd, 50)  # 301^3, step 0.1
            energies = -0.5 * rng.uniform(0.5, 2.0, nd) ** 2  # kappa ~ U[0.5, 2]
        step = 0.2 if wl == "gbfmm_batch_256" else 0.1
        grids, rhos, outs = [], [], []
        inject_ms = None
        if wl == "helmholtz_step_301":
            bub, gcube = _molecule_bubbles(dage, rng)
            base = torch.zeros(301 ** 3, dtype=torch.float64, device=dev)
            inject_ms = _timed(lambda: bub.inject(gcube, cube=base.zero_()), args.steps,
                               args.warmup, sync)
        for i in range(nd):
            nc = int(cells[i])
            half = 0.5 * nc * 6 * step
            grids.append(dage.Grid3D.cube(-half, nc, step))
            ng = int(rng.integers(1, 9))
            q, a = rng.uniform(-1, 2, ng), rng.uniform(0.3, 6, ng)
            c = rng.uniform(-0.6 * half, 0.6 * half, (ng, 3))
            rho = _gauss_cube(dev, nc, step, q, a, c)
            if wl == "helmholtz_step_301":
                rho += rng.uniform(0.5, 1.5) * base  # the injected bubbles of the molecule
            rhos.append(rho)
            outs.append(torch.empty_like(rho))
        quad = dage.GaussQuad(20, 20, 0.0, TLIN, TLOG)
        prec = "fp64" if args.precision == "fp64" else "fp16x3"
        bt = dage.GBFMMBatch(grids, lmax=lmax, quad=quad, precision=prec)
        if energies is not None:
            bt.set_energies(energies)
        Ebox = {}
        clk.start()
        ms = _timed(lambda: Ebox.update(e=bt.apply(rhos, outs, energy=True)), args.steps,
                    args.warmup, sync)
        clocks = clk.stop()
        nplans, nchunks, tiles, nodes = bt.info()
        # per-density check of a few densities against the single-density operator
        chk = []
        for i in range(3):
            op = (dage.GBFMMHelmholtz3D(grids[i], energies[i], lmax=lmax, quad=quad, precision=prec)
                  if energies is not None else
                  dage.GBFMMCoulomb3D(grids[i], lmax=lmax, quad=quad, precision=prec))
            V1 = torch.empty_like(rhos[i])
            op.apply(rhos[i], out=V1)
            chk.append(float((outs[i] - V1).abs().max() / V1.abs().max()))
            del op
        pts = float(sum(int(gr.shape[0]) ** 3 for gr in grids))
        metric = ("GBFMM batch Mpts/s, 256 densities 61^3..181^3, %s, lmax 12"
                  if wl == "gbfmm_batch_256" else
                  "Helmholtz GBFMM batch Mpts/s, 64 orbitals 301^3, %s, lmax 10") % (
                      "FP64" if prec == "fp64" else "fp16x3 near field")
        extra = {"per_density_check": {"vs": "single-density operator", "max_rel": max(chk)},
                 "batch": {"densities": nd, "plans": nplans,
                           "near_chunks" if prec == "fp64" else "near_sets": nchunks,
                           "tiles": list(tiles), "graph_nodes": nodes}}
        if prec != "fp64":
            # the FP64 batch on the same densities: per-instance errors of the
            # split precision and the FP64 time
            E16 = Ebox["e"]
            del bt
            torch.cuda.empty_cache()
            b64 = dage.GBFMMBatch(grids, lmax=lmax, quad=quad)
            if energies is not None:
                b64.set_energies(energies)
            outs64 = [torch.empty_like(r) for r in rhos]
            E64box = {}
            ms64 = _timed(lambda: E64box.update(e=b64.apply(rhos, outs64, energy=True)), 1, 1, sync)
            E64 = E64box["e"]
            vmax, vrms, erel = [], [], []
            for i in range(nd):
                d = (outs[i] - outs64[i]).abs()
                s64 = outs64[i].abs().max()
                vmax.append(float(d.max() / s64))
                vrms.append(float(d.pow(2).mean().sqrt() / s64))
                erel.append(abs(E16[i] - E64[i]) / abs(E64[i]))
            w = int(np.argmax(erel))
            # cancellation of the worst instance: |int rho V| / int |rho V|
            absE = dage.integrate(grids[w], rhos[w].abs(), outs64[w].abs())
            extra["mixed_vs_fp64"] = {
                "per_instance_max_rel": {"max": max(vmax), "median": float(np.median(vmax))},
                "per_instance_rms_rel": {"max": max(vrms), "median": float(np.median(vrms))},
                "per_instance_energy_rel": {"max": max(erel), "median": float(np.median(erel))},
                "instances_over_bars": {"potential_1e-6": int(sum(v > 1e-6 for v in vmax)),
                                        "energy_1e-7": int(sum(e > 1e-7 for e in erel))},
                "worst_energy_instance": {"index": w, "points_per_axis": int(grids[w].shape[0]),
                                          "energy_rel": erel[w],
                                          "abs_energy_over_int_abs_rho_V": abs(E64[w]) / absE},
                "fp64_ms_per_step": ms64, "speedup_vs_fp64": ms64 / ms}
            del b64, outs64
        if inject_ms is not None:
            extra["bubbles_inject"] = {"ms": inject_ms, "atoms": 20, "lmax": 2,
                                       "points": 301 ** 3,
                                       "Mpts_per_s": 301 ** 3 / inject_ms / 1e3}
        _line(args, world, metric, pts / ms / 1e3, "Mpts/s", ms, "f64" if prec == "fp64" else "f16",
              {"workload": wl, "densities": nd, "step_bohr": step, "t_points": 40,
               "lmax": lmax, "boxes": 64, "seed": SEED, "precision": prec,
               "sizes": sorted(set(int(6 * x + 1) for x in cells))}, clocks, nodes, extra)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=10)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="dage", choices=["dage", "reference"])
    ap.add_argument("--precision", default=os.environ.get("DAGE_BENCH_PRECISION", "fp16x3"),
                    choices=["fp64", "bf16x3", "bf16x6", "fp16x3"])
    ap.add_argument("--fp64-steps", type=int, default=5)
    ap.add_argument("--skip-fp64", action="store_true")
    ap.add_argument("--skip-cpu", action="store_true")
    ap.add_argument("--skip-e2e", action="store_true")
    ap.add_argument("--skip-alt", action="store_true", help="do not time the other split-precision mode")
    ap.add_argument("--n-cell", type=int, default=N_CELL,
                    help="cells per axis (80 -> 481^3, the headline workload)")
    ap.add_argument("--workload", default="coulomb_cube_481",
                    choices=["coulomb_cube_481", "coulomb_cube_121", "gbfmm_241", "gbfmm_241_adaptive", "helmholtz_gbfmm_241",
                             "gbfmm_batch_256", "helmholtz_step_301", "bubbles_inject_301",
                             "density_product_301"],
                    help="coulomb_cube_481 is the headline line; the others time the other "
                         "configurations of the path")
    args = ap.parse_args()
    world, rank, local = dist_setup()
    try:
        if args.impl == "reference":
            run_reference(args, world, rank)
        elif args.workload != "coulomb_cube_481":
            run_workload(args, world, rank, local)
        else:
            run_gpu(args, world, rank, local)
    finally:
        if world > 1:
            import torch.distributed as dist

            dist.destroy_process_group()


if __name__ == "__main__":
    main()

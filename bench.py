"""Benchmark: the fixed-source DG1 SN solve on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step is one full solve, from zero, of the 256 x 256 jittered-triangle DG1
S8 one-group problem (15.7M unknowns) to a true relative residual of 1e-8,
plain FP64, with the right-hand side resident in HBM: the reference's plain
FP64 drop-in configuration. `value` is seconds per solve (lower is better).
Beside it the line carries the mixed FP32+FP64-refinement solve, the adjoint
gradient of the detector response (same mesh), the operator apply in GB/s,
the roofline of the dominant kernel, the CPU restatement timed on this host's
cores, the end-to-end solve through the public API with host buffers, the SM
clocks seen during the timed region and the library's kernel launch count.

Multi-GPU: replicas only - each rank solves its own copy (the solve is not
sharded); value aggregates the solves of all ranks per second of the slowest
rank's time, reported as seconds per solve per replica set.

--impl reference times the reference path's CPU restatement (the oracle port:
the reference build needs PETSc + Kokkos + PFLARE, which are not installed) on
all host cores, on the same workload; other ranks exit without work.
"""
import argparse
import json
import os
import sys
import threading
import time

# The CPU legs run OpenMP on every host core, threads kept close to their
# parent; set before any OpenMP runtime starts in this process
os.environ.setdefault("OMP_PROC_BIND", "close")

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "solve s to 1e-8 resid, FP32+refine vs FP64 on 1 B200; adjoint grad s; apply GB/s"
WORKLOAD = "tri256_dg1_s8: 2D DG1, 256x256 jittered quads split into 131072 triangles, S8 (40 ordinates), 1 group"


def _args():
    p = argparse.ArgumentParser()
    p.add_argument("--gpus", type=int, default=1)
    p.add_argument("--steps", type=int, default=10)
    p.add_argument("--warmup", type=int, default=3)
    p.add_argument("--impl", default="ours", choices=["ours", "reference"])
    p.add_argument("--scale", type=float, default=1.0, help="mesh scale (1.0 = the named workload)")
    p.add_argument("--no-cpu-baseline", action="store_true")
    p.add_argument("--quick", action="store_true", help="skip the secondary measurements")
    p.add_argument("--no-workloads", action="store_true",
                   help="skip the hex128 and tet44 solve configurations that follow the headline")
    p.add_argument("--reps", type=int, default=2, help="timed repetitions of each hex128 / tet44 measurement")
    p.add_argument("--workload", default="tri256", choices=["tri256", "hex128", "tet44"],
                   help="tri256 is the headline line; hex128 (4 groups) and tet44 time the other solve configs")
    p.add_argument("--restart", type=int, default=0, help="GMRES restart (0: 30, or 10 for hex128)")
    p.add_argument("--profile", default="",
                   choices=["", "apply", "apply32", "sweep", "sweep32", "sweep_iso", "sweep_iso32", "wave", "wave32", "adjoint", "adjoint32",
                            "dsa_spmv", "block", "gradient", "scalar_flux"],
                   help="run only this kernel, --warmup + --steps launches on the workload, for a profiler")
    return p.parse_args()


def _peaks():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """SM clock, power and clock-event reasons sampled through NVML every
    10 ms while the timed region runs (read only; nothing is set)."""

    def __init__(self, index=0):
        self.index = index
        self.samples = []
        self.stop = threading.Event()
        self.thread = None

    def __enter__(self):
        try:
            import pynvml as nv
            nv.nvmlInit()
            self.nv = nv
            self.h = nv.nvmlDeviceGetHandleByIndex(self.index)
            self.max_sm = nv.nvmlDeviceGetMaxClockInfo(self.h, nv.NVML_CLOCK_SM)
            self.thread = threading.Thread(target=self._run, daemon=True)
            self.thread.start()
        except Exception:
            self.thread = None
        return self

    def _run(self):
        nv = self.nv
        while not self.stop.is_set():
            try:
                sm = nv.nvmlDeviceGetClockInfo(self.h, nv.NVML_CLOCK_SM)
                reasons = nv.nvmlDeviceGetCurrentClocksEventReasons(self.h)
                power = nv.nvmlDeviceGetPowerUsage(self.h) / 1e3
                self.samples.append((sm, reasons, power))
            except Exception:
                pass
            self.stop.wait(0.01)

    def __exit__(self, *a):
        if self.thread:
            self.stop.set()
            self.thread.join(timeout=5)
            try:
                self.nv.nvmlShutdown()
            except Exception:
                pass

    def summary(self):
        if not self.samples:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        nv = self.nv
        bits = {"hw_slowdown": nv.nvmlClocksEventReasonHwSlowdown,
                "hw_thermal_slowdown": nv.nvmlClocksEventReasonHwThermalSlowdown,
                "sw_thermal_slowdown": nv.nvmlClocksEventReasonSwThermalSlowdown,
                "sw_power_cap": nv.nvmlClocksEventReasonSwPowerCap}
        reasons = sorted({k for _, r, _ in self.samples for k, b in bits.items() if r & b})
        return {"sm_mhz": float(np.median([s for s, _, _ in self.samples])), "sm_max_mhz": float(self.max_sm),
                "reasons": reasons, "samples": len(self.samples),
                "power_w_median": float(np.median([p for _, _, p in self.samples]))}


def max_over_ranks(v, world, device):
    """The slowest rank's value (every rank takes part; world 1: v itself)."""
    if world == 1:
        return v
    import torch
    import torch.distributed as dist
    t = torch.tensor([v], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replica_seconds_per_solve(ms_per_step, world):
    """Replicas: each rank solves its own copy per step, so the job finishes
    `world` solves per (slowest rank's) step: seconds per solve of the job."""
    return ms_per_step / 1e3 / world


def _dist():
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return world, rank, local


def cpu_model():
    try:
        with open("/proc/cpuinfo") as fh:
            for line in fh:
                if line.startswith("model name"):
                    return line.split(":", 1)[1].strip()
    except OSError:
        pass
    return "unknown"


def run_reference(args):
    """The CPU restatement of the reference path on every host core. The
    workload's mesh and seeded data come from the library's pure-NumPy
    builders, its geometry and ordinates from the oracle: the library itself
    is never loaded here."""
    world, rank, _ = _dist()
    if rank != 0:
        return
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from ubolt_b200 import problem as P
    prob = P.config_tri256(scale=args.scale, geometry=O.geometry_from_mesh, quadrature=O.lqn)
    g, q = prob.geometry, prob.quad
    op = O.Operator(g, q, prob.sigma_t[0], prob.sigma_s[0, 0])
    b = O.rhs(g, q, prob.source[0])
    for _ in range(args.warmup):
        op.solve(b, rtol=1e-8)
    times, its = [], []
    for _ in range(args.steps):
        t0 = time.perf_counter()
        x, it, res = op.solve(b, rtol=1e-8)
        times.append(time.perf_counter() - t0)
        its.append(it)
    v = float(np.mean(times))
    cores = O.threads()
    line = {"metric": METRIC, "value": v, "unit": "s/solve", "n_gpus": args.gpus, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": v * 1e3, "higher_is_better": False, "scaling": "weak",
            "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded)", "impl": "reference",
            "config": {"workload": WORKLOAD, "rtol": 1e-8, "rows": int(op.n), "iterations": int(np.median(its)),
                       "parallelism": f"replicas{args.gpus}"},
            "cpu_baseline": {"value": v, "unit": "s/solve", "cores": cores, "kind": "port",
                             "cpu_model": cpu_model(), "omp_proc_bind": os.environ.get("OMP_PROC_BIND"),
                             "sample": "the full workload: one FP64 GMRES solve to 1e-8 with an upwind-sweep "
                                       "preconditioner per step, OpenMP on every host core"},
            "e2e": {"value": v, "unit": "s/solve", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def cpu_baseline(args):
    sys.path.insert(0, os.path.join(ROOT, "oracle"))
    import oracle as O
    from ubolt_b200 import problem as P
    prob = P.config_tri256(scale=args.scale)
    g, q = prob.geometry, prob.quad
    op = O.Operator(g, q, prob.sigma_t[0], prob.sigma_s[0, 0])
    b = O.rhs(g, q, prob.source[0])
    op.solve(b, rtol=1e-8)
    t0 = time.perf_counter()
    n = 2
    for _ in range(n):
        x, it, res = op.solve(b, rtol=1e-8)
    v = (time.perf_counter() - t0) / n
    return {"value": v, "unit": "s/solve", "cores": O.threads(), "kind": "port", "cpu_model": cpu_model(),
            "omp_proc_bind": os.environ.get("OMP_PROC_BIND"),
            "sample": f"the full workload, {n} FP64 solves to 1e-8 ({it} iterations each), GMRES + CPU upwind "
                      "sweep, OpenMP, on the oracle's own geometry and ordinates"}, x


def profile_kernel(args, ctx, T, stream):
    """--profile: one kernel alone on the workload, timed with CUDA events."""
    import torch
    dt = torch.float32 if args.profile.endswith("32") else torch.float64
    g = torch.Generator(device="cuda").manual_seed(7)
    xr = torch.rand(ctx.n_rows, dtype=torch.float64, device="cuda", generator=g).to(dt)
    yr = torch.empty_like(xr)
    kind = args.profile.rstrip("32")
    if kind in ("sweep", "wave"):
        sw = T.Sweep(ctx, 0)
        sw.set_kernel("tasks" if kind == "sweep" else "wave")
        fn = lambda: sw.apply(xr, yr)
    elif kind == "sweep_iso":
        sw = T.Sweep(ctx, 0)
        sw.set_kernel("tasks")
        phr = torch.rand(ctx.n_nodes, dtype=torch.float64, device="cuda", generator=g)
        fn = lambda: sw.apply_iso(phr, yr, ordinate_major=True)
    elif kind == "dsa_spmv":
        dsa = T.DSAPrecon(ctx)
        dsa.set_group()
        u = dsa.restrict(xr)
        v = torch.empty_like(u)
        fn = lambda: dsa.spmv(u, v)
    elif kind == "block":
        blk = T.ElementBlockInverse(ctx)
        fn = lambda: blk.apply(xr, yr)
    elif kind == "gradient":
        lam = torch.rand_like(xr)
        fn = lambda: T.gradient(ctx, xr, lam)
    elif kind == "scalar_flux":
        phi = torch.empty(ctx.n_nodes, dtype=xr.dtype, device="cuda")
        fn = lambda: T.angular_integral(ctx, xr, phi)
    else:
        A = T.TransportOperator(ctx)
        fn = (lambda: A.mult(xr, yr)) if kind == "apply" else (lambda: A.mult_transpose(xr, yr))
    for _ in range(args.warmup):
        fn()
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        fn()
    e1.record(stream)
    torch.cuda.synchronize()
    print(json.dumps({"profile": args.profile, "workload": WORKLOAD, "launches": args.steps,
                      "us_per_launch": e0.elapsed_time(e1) / args.steps * 1e3}), flush=True)


def _events_ms(fn, stream, reps=1, warm=1):
    """Median milliseconds of fn() over reps runs, CUDA events on `stream`."""
    import torch
    for _ in range(warm):
        fn()
    torch.cuda.synchronize()
    out = []
    for _ in range(reps):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        fn()
        e1.record(stream)
        torch.cuda.synchronize()
        out.append(e0.elapsed_time(e1))
    return float(np.median(out))


def kernel_map(ctx, T, prob, stream, peak, peak_kind):
    """Every kernel of the path on the workload, alone, with CUDA events: its
    time, the algorithmic bytes of one launch (ψ in and out, cross sections;
    geometry and indices excluded, so the figure never exceeds what must
    move) over that time, and the fraction of the measured copy bandwidth."""
    import torch
    n, nc, nn, nb = ctx.n_rows, ctx.n_cells, ctx.n_nodes, prob.geometry.n_basis
    F = prob.geometry.faces_per_cell
    g = torch.Generator(device="cuda").manual_seed(11)
    x64 = torch.rand(n, dtype=torch.float64, device="cuda", generator=g)
    y64 = torch.empty_like(x64)
    x32, y32 = x64.float(), torch.empty(n, dtype=torch.float32, device="cuda")
    phi = torch.rand(nn, dtype=torch.float64, device="cuda", generator=g)
    src = torch.rand(nc, dtype=torch.float64, device="cuda", generator=g)
    A = T.TransportOperator(ctx)
    B = T.ElementBlockInverse(ctx)
    B.setup()
    sw = T.Sweep.__new__(T.Sweep)
    sw.ctx = ctx
    ss = torch.tensor(prob.sigma_s[0, 0], device="cuda")
    tr = T.GroupTransfer(ctx, [[ss, ss], [ss, ss]], [src, src])
    tr.phi = [phi, phi]
    dsa = T.DSAPrecon(ctx)
    dsa.set_group()
    u = torch.rand(nn, dtype=torch.float64, device="cuda", generator=g)
    lam = torch.rand(n, dtype=torch.float64, device="cuda", generator=g)
    nnz = nc * (F + 1) * nb * nb
    cases = {
        "apply_fp64": (lambda: A.mult(x64, y64), 2 * n * 8 + 2 * nc * 8),
        "apply_fp32": (lambda: A.mult(x32, y32), 2 * n * 4 + 2 * nc * 4),
        "apply_unscattered_fp64": (lambda: A.mult_unscattered(x64, y64), 2 * n * 8 + nc * 8),
        "apply_adjoint_fp64": (lambda: A.mult_transpose(x64, y64), 2 * n * 8 + 2 * nc * 8),
        "block_apply_fp64": (lambda: B.apply(x64, y64), 2 * n * 8 + nc * 8),
        "sweep_fp64": (lambda: sw.apply(x64, y64), 2 * n * 8 + nc * 8),
        "sweep_fp32": (lambda: sw.apply(x32, y32), 2 * n * 4 + nc * 4),
        "scalar_flux_fp64": (lambda: T.angular_integral(ctx, x64, phi), n * 8 + nn * 8),
        "add_transfer_fp64": (lambda: tr.add_transfer(0, 1, y64), 2 * n * 8 + nn * 8 + nc * 8),
        "dsa_restrict_fp64": (lambda: dsa.restrict(x64), n * 8 + nn * 8),
        "dsa_prolong_fp64": (lambda: dsa.prolong(u), n * 8 + nn * 8),
        "dsa_spmv_fp64": (lambda: dsa.spmv(u), nnz * 8 + 2 * nn * 8),
        "gradient_fp64": (lambda: T.gradient(ctx, x64, lam), 2 * n * 8 + 2 * nc * 8),
    }
    out = {}
    for name, (fn, nbytes) in cases.items():
        ms = _events_ms(lambda: [fn() for _ in range(10)], stream, reps=3, warm=1) / 10
        gbs = nbytes / (ms * 1e-3) / 1e9
        out[name] = {"us": ms * 1e3, "bytes": int(nbytes), "gbs": gbs, "frac": gbs / peak}
    out["_peak"] = {"gbs": peak, "source": peak_kind}
    return out


def workload_hex128(args, stream):
    """The mixed-precision configuration: 128^3 hexes, DG1, S8, 4 downscatter
    groups; FP64 and FP32+refinement group solves to 1e-8, medians of
    args.reps after a warm-up."""
    import torch
    from ubolt_b200 import problem as P
    from ubolt_b200 import transport as T
    t0 = time.perf_counter()
    prob = P.config_hex128(scale=args.scale)
    ctx = T.Context(prob.geometry, prob.quad)
    out = {"workload": prob.name + ": 128^3 hex box, DG1 (4 modes), S8 (80 ordinates), 4 groups, downscatter",
           "rows_per_group": ctx.n_rows, "restart": 10, "setup_s": time.perf_counter() - t0}
    phis = {}
    # Inputs resident and solvers set up before the timed region, as the
    # reference's group loop sets up once and reuses
    tables = T.group_tables(ctx, prob.sigma_t, prob.sigma_s, prob.source)
    for precision in ("fp64", "mixed"):
        t1 = time.perf_counter()
        solver = T.TransportSolver(ctx, rtol=prob.rtol, precision=precision, pc="sweep", restart=10, max_it=500)
        torch.cuda.synchronize()
        out.setdefault("solver_setup_s", {})[precision] = time.perf_counter() - t1
        res = {}

        def run():
            res["phi"], res["stats"] = T.solve_groups(ctx, *tables, solver=solver)

        ms = _events_ms(run, stream, reps=args.reps, warm=1)
        st = res["stats"]
        phis[precision] = [p_.clone() for p_ in res["phi"]]
        out[precision] = {"s_per_solve": ms / 1e3, "iterations": [s_["iterations"] for s_ in st],
                          "outer": [s_["outer"] for s_ in st], "residual": max(s_["residual"] for s_ in st)}
    out["mixed"]["phi_rel_err_vs_fp64"] = max(float((m - f).norm() / f.norm())
                                              for m, f in zip(phis["mixed"], phis["fp64"]))
    out["mixed"]["speedup_vs_fp64"] = out["fp64"]["s_per_solve"] / out["mixed"]["s_per_solve"]
    sw = T.Sweep.__new__(T.Sweep)
    sw.ctx = ctx
    xr = torch.rand(ctx.n_rows, dtype=torch.float64, device="cuda")
    yr = torch.empty_like(xr)
    out["sweep_ms"] = {"fp64": _events_ms(lambda: sw.apply(xr, yr), stream, reps=3)}
    del xr, yr
    xf = torch.rand(ctx.n_rows, dtype=torch.float32, device="cuda")
    yf = torch.empty_like(xf)
    out["sweep_ms"]["fp32"] = _events_ms(lambda: sw.apply(xf, yf), stream, reps=3)
    del xf, yf
    info = sw.status()
    out["sweep"] = {k: info[k] for k in ("n_tasks", "n_split", "n_lagged", "factor_bytes", "patch_size", "kernel")}
    ctx.close()
    return out


def workload_tet44(args, stream):
    """The combined configuration: 511,104 jittered Kuhn tets, DG1, S8 3D, one
    group, diffusive: FP64 and mixed forward solves, sweep + DSA against the
    sweep alone, and the adjoint gradient of a detector response with respect
    to the per-cell cross sections through the mixed form."""
    import torch
    from ubolt_b200 import problem as P
    from ubolt_b200 import transport as T
    t0 = time.perf_counter()
    prob = P.config_tet44(scale=args.scale)
    ctx = T.Context(prob.geometry, prob.quad)
    st = torch.tensor(prob.sigma_t[0], device="cuda")
    ss = torch.tensor(prob.sigma_s[0, 0], device="cuda")
    ctx.set_group(st, ss)
    src = torch.tensor(prob.source[0], device="cuda")
    b = ctx.vector(fill=0.0)
    T.GroupTransfer(ctx, [[ss]], [src]).add_external(0, b)
    out = {"workload": prob.name + ": 44^3 cubes in Kuhn tets (jittered), DG1 (4 modes), S8 (80 ordinates), 1 group",
           "rows": ctx.n_rows, "setup_s": time.perf_counter() - t0}
    xs = {}
    for key, opts in (("fp64", dict(precision="fp64", pc="sweep")), ("mixed", dict(precision="mixed", pc="sweep")),
                      ("fp64_dsa", dict(precision="fp64", pc="sweep+dsa"))):
        solver = T.TransportSolver(ctx, rtol=prob.rtol, restart=30, max_it=500, **opts)
        if key == "fp64_dsa":
            dsa = T.DSAPrecon(ctx)
            dsa.set_group()
        x = ctx.vector(fill=0.0)
        res = {}

        def run():
            res["x"], res["stats"] = solver.solve(b, x)

        ms = _events_ms(run, stream, reps=args.reps, warm=1)
        xs[key] = res["x"].clone()
        out[key] = {"s_per_solve": ms / 1e3, "iterations": res["stats"]["iterations"],
                    "residual": res["stats"]["residual"]}
    phi64 = T.angular_integral(ctx, xs["fp64"])
    out["mixed"]["phi_rel_err_vs_fp64"] = float((T.angular_integral(ctx, xs["mixed"]) - phi64).norm() / phi64.norm())
    out["mixed"]["speedup_vs_fp64"] = out["fp64"]["s_per_solve"] / out["mixed"]["s_per_solve"]
    out["fp64_dsa"]["phi_rel_err_vs_fp64"] = float((T.angular_integral(ctx, xs["fp64_dsa"]) - phi64).norm()
                                                   / phi64.norm())
    out["fp64_dsa"]["speedup_vs_sweep_only"] = out["fp64"]["s_per_solve"] / out["fp64_dsa"]["s_per_solve"]
    # Adjoint gradient through the mixed form
    det = P.detector_patch(prob, cells_per_side=11, seed_index=4).astype(np.float64)
    model = T.DetectorResponse(ctx, prob.source[0], det, rtol=prob.rtol, max_it=500, precision="mixed")
    sig_t = st.clone().requires_grad_(True)
    sig_s = ss.clone().requires_grad_(True)
    J = model(sig_t, sig_s)
    torch.autograd.grad(J, (sig_t, sig_s))
    torch.cuda.synchronize()
    g0, g1, g2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
    g0.record(stream)
    J = model(sig_t, sig_s)
    g1.record(stream)
    gt, gs = torch.autograd.grad(J, (sig_t, sig_s))
    g2.record(stream)
    torch.cuda.synchronize()
    fwd, tot = g0.elapsed_time(g1), g0.elapsed_time(g2)
    out["adjoint"] = {"grad_s": tot / 1e3, "forward_s": fwd / 1e3, "adjoint_over_forward": (tot - fwd) / fwd,
                      "precision": "mixed", "parameters": 2 * ctx.n_cells, "J": float(J.item()),
                      "adjoint_iterations": model.last_adjoint["iterations"],
                      "detector_cells": int(det.sum())}
    ctx.set_group(st, ss)
    ctx.close()
    return out


def workload_cg256(args, stream):
    """The CG-SUPG backend at the named problem's size: 256 x 256 jittered
    quads (66,049 vertices), S8, one group, the config-1 cross-section law
    per element; GMRES with point Jacobi, and with the vertex DSA stage, FP64
    and mixed, to 1e-8; the SUPG operator apply alone."""
    import torch
    from ubolt_b200 import problem as P
    from ubolt_b200 import transport as T
    t0 = time.perf_counter()
    n = max(4, int(round(256 * args.scale)))
    s_mesh, s_xs, _, _ = P._streams(6)
    mesh = P.box_quads(n, n, jitter=0.2, rng=s_mesh)
    g = P.build_cg_geometry(mesh)
    q = P.lqn(2, 8)
    ne = g.n_elements
    st = s_xs.lognormal(0.0, 0.5, ne)
    ss = st * s_xs.uniform(0.3, 0.99, ne)
    ctx = T.Context(g, q)
    keep = (torch.tensor(st, device="cuda"), torch.tensor(ss, device="cuda"))
    ctx.set_group(*keep)
    b = ctx.vector(fill=0.0)
    src = torch.ones(ne, dtype=torch.float64, device="cuda")
    from ubolt_b200 import _lib
    _lib.check(_lib.lib.ubolt_add_source(ctx.handle, T._p(src), T._p(b), T._stream()))
    out = {"workload": f"cg{n}_s8: CG-SUPG (Q1) on {n}x{n} jittered quads, {g.n_vertices} vertices, S8, 1 group",
           "rows": ctx.n_rows, "setup_s": time.perf_counter() - t0}
    xs = {}
    for key, opts in (("jacobi_fp64", dict(precision="fp64", pc="block")),
                      ("jacobi_dsa_fp64", dict(precision="fp64", pc="block+dsa")),
                      ("jacobi_dsa_mixed", dict(precision="mixed", pc="block+dsa"))):
        if "dsa" in key:
            dsa = T.DSAPrecon(ctx)
            dsa.set_group()
        solver = T.TransportSolver(ctx, rtol=1e-8, restart=60, max_it=3000, **opts)
        x = ctx.vector(fill=0.0)
        res = {}

        def run():
            res["x"], res["stats"] = solver.solve(b, x)

        ms = _events_ms(run, stream, reps=args.reps, warm=1)
        xs[key] = res["x"].clone()
        out[key] = {"s_per_solve": ms / 1e3, "iterations": res["stats"]["iterations"],
                    "residual": res["stats"]["residual"]}
    phi = T.angular_integral(ctx, xs["jacobi_fp64"])
    for key in ("jacobi_dsa_fp64", "jacobi_dsa_mixed"):
        out[key]["phi_rel_err_vs_jacobi_fp64"] = float((T.angular_integral(ctx, xs[key]) - phi).norm() / phi.norm())
    A = T.TransportOperator(ctx)
    xr = torch.rand(ctx.n_rows, dtype=torch.float64, device="cuda")
    yr = torch.empty_like(xr)
    us = _events_ms(lambda: A.mult(xr, yr), stream, reps=20, warm=3) * 1e3
    byts = 2 * ctx.n_rows * 8 + 2 * ne * 8
    out["apply_fp64"] = {"us": us, "bytes": byts, "gbs": byts / us / 1e3}
    ctx.close()
    return out


def workload_upscatter(args, stream):
    """The upscatter outer iteration: the 128 x 128 triangle mesh of the
    named problem's family, DG1, S8, three groups with thermal upscatter
    (2 -> 1), block Gauss-Seidel over the thermal block to an error
    estimate of 1e-8, with the angular and the moments store."""
    import torch
    from ubolt_b200 import problem as P
    from ubolt_b200 import transport as T
    n = max(4, int(round(128 * args.scale)))
    s_mesh, s_xs, _, _ = P._streams(7)
    mesh = P.box_tris(n, n, jitter=0.2, rng=s_mesh, tile=8, diagonals="random")
    g = P.build_geometry(mesh, 1)
    q = P.lqn(2, 8)
    nc, G = g.n_cells, 3
    st = s_xs.lognormal(0.0, 0.5, (G, nc))
    ss = np.zeros((G, G, nc))
    for gg in range(G):
        ss[gg, gg] = 0.5 * st[gg]
    ss[0, 1], ss[0, 2], ss[1, 2] = 0.2 * st[0], 0.1 * st[0], 0.25 * st[1]
    ss[2, 1] = 0.3 * st[2]
    src = np.zeros((G, nc))
    src[0] = 1.0
    ctx = T.Context(g, q)
    tables = T.group_tables(ctx, st, ss, src)
    solver = T.TransportSolver(ctx, rtol=1e-8, restart=30, max_it=500)
    out = {"workload": f"tri{n}_s8_g3_up: 2D DG1, {nc} triangles, S8, 3 groups, thermal upscatter 2 -> 1",
           "rows_per_group": ctx.n_rows}
    for store in ("angular", "moments"):
        info = {}
        res = {}

        def run():
            info.clear()
            res["phis"], _ = T.solve_groups(ctx, *tables, solver=solver, outer_rtol=1e-8, outer_store=store,
                                            outer_info=info)

        ms = _events_ms(run, stream, reps=max(1, args.reps), warm=1)
        out[store] = {"s_per_solve": ms / 1e3, "outer_iterations": info.get("outer_iterations"),
                      "error_estimate": info.get("error_estimate"), "converged": info.get("converged")}
    ctx.close()
    return out


def run_workload(args):
    """--workload hex128 | tet44: the other solve configs, FP64 and mixed, as one
    JSON line each (no CPU baseline: the restatement would take hours here)."""
    import torch
    from ubolt_b200 import problem as P
    from ubolt_b200 import transport as T
    torch.cuda.set_device(0)
    t0 = time.perf_counter()
    prob = P.CONFIGS[args.workload](scale=args.scale)
    ctx = T.Context(prob.geometry, prob.quad)
    setup_s = time.perf_counter() - t0
    restart = args.restart or (10 if args.workload == "hex128" else 30)
    out = {"workload": prob.name, "cells": prob.geometry.n_cells, "ordinates": prob.quad.n_angles,
           "n_basis": prob.geometry.n_basis, "groups": prob.n_groups, "rows_per_group": ctx.n_rows,
           "restart": restart, "setup_s": setup_s}
    phis = {}
    tables = T.group_tables(ctx, prob.sigma_t, prob.sigma_s, prob.source)
    for precision in ("fp64", "mixed"):
        solver = T.TransportSolver(ctx, rtol=prob.rtol, precision=precision, pc="sweep", restart=restart,
                                   max_it=500)
        stream = torch.cuda.current_stream()
        for rep in range(1 + args.steps):
            e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            e0.record(stream)
            phi, stats = T.solve_groups(ctx, *tables, solver=solver)
            e1.record(stream)
            torch.cuda.synchronize()
            if rep == 0:
                times = []
                continue
            times.append(e0.elapsed_time(e1) / 1e3)
        phis[precision] = [p.clone() for p in phi]
        out[precision] = {"s_per_solve": float(np.median(times)),
                          "iterations": [s_["iterations"] for s_ in stats],
                          "residual": max(s_["residual"] for s_ in stats),
                          "krylov": [{1: "full", 2: "compressed"}.get(s_["krylov"]) for s_ in stats]}
    err = max(float((m - f).norm() / f.norm()) for m, f in zip(phis["mixed"], phis["fp64"]))
    out["mixed"]["phi_rel_err_vs_fp64"] = err
    out["mixed"]["speedup_vs_fp64"] = out["fp64"]["s_per_solve"] / out["mixed"]["s_per_solve"]
    sw = T.Sweep.__new__(T.Sweep)
    sw.ctx = ctx
    out["sweep"] = {k: v for k, v in sw.status().items() if k in ("n_tasks", "n_lagged", "n_split", "factor_bytes")}
    print(json.dumps(out), flush=True)
    ctx.close()


def main():
    args = _args()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload != "tri256":
        run_workload(args)
        return
    import torch
    import torch.distributed as dist
    from ubolt_b200 import _lib
    from ubolt_b200 import problem as P
    from ubolt_b200 import transport as T

    world, rank, local = _dist()
    torch.cuda.set_device(local)
    if world > 1:
        dist.init_process_group("nccl", init_method="env://", timeout=__import__("datetime").timedelta(seconds=120),
                                device_id=torch.device("cuda", local))

    def barrier():
        if world > 1:
            dist.barrier()


    prob = P.config_tri256(scale=args.scale)
    g, q = prob.geometry, prob.quad
    ctx = T.Context(g, q)
    st = torch.tensor(prob.sigma_t[0], device="cuda")
    ss = torch.tensor(prob.sigma_s[0, 0], device="cuda")
    ctx.set_group(st, ss)
    src = torch.tensor(prob.source[0], device="cuda")
    b = ctx.vector(fill=0.0)
    T.GroupTransfer(ctx, [[ss]], [src]).add_external(0, b)
    n = ctx.n_rows
    if args.profile:
        profile_kernel(args, ctx, T, stream=torch.cuda.current_stream())
        ctx.close()
        return
    t_setup = time.perf_counter()
    solver = T.TransportSolver(ctx, rtol=1e-8, precision="fp64", pc="sweep", restart=30, max_it=500)
    setup_s = time.perf_counter() - t_setup
    stream = torch.cuda.current_stream()
    x = ctx.vector(fill=0.0)

    # ~~~ Headline: plain FP64 solve, inputs resident
    for _ in range(args.warmup):
        solver.solve(b, x)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches0 = _lib.lib.ubolt_launch_count()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    with Clocks(local) as clk:
        e0.record(stream)
        for _ in range(args.steps):
            x, st_ = solver.solve(b, x)
            stats.append(st_)
        e1.record(stream)
        torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    launches = (_lib.lib.ubolt_launch_count() - launches0)
    ms = max_over_ranks(e0.elapsed_time(e1) / args.steps, world, "cuda")
    value = replica_seconds_per_solve(ms, world)
    its = int(np.median([s["iterations"] for s in stats]))
    res = float(max(s["residual"] for s in stats))

    extra = {}
    if not args.quick:
        # ~~~ Kernel timings: apply (FP64, FP32), sweep (FP64, FP32)
        A = T.TransportOperator(ctx)
        sw = T.Sweep.__new__(T.Sweep)
        sw.ctx = ctx
        def timed(fn, reps=20):
            for _ in range(3):
                fn()
            torch.cuda.synchronize()
            a0, a1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a0.record(stream)
            for _ in range(reps):
                fn()
            a1.record(stream)
            torch.cuda.synchronize()
            return a0.elapsed_time(a1) / reps
        xr = torch.randn(n, dtype=torch.float64, device="cuda")
        yr = torch.empty_like(xr)
        xf, yf = xr.float(), torch.empty(n, dtype=torch.float32, device="cuda")
        t_apply64 = timed(lambda: A.mult(xr, yr))
        t_apply32 = timed(lambda: A.mult(xf, yf))
        t_sweep64 = timed(lambda: sw.apply(xr, yr))
        t_sweep32 = timed(lambda: sw.apply(xf, yf))
        # The form the compressed solve runs every iteration: an isotropic
        # source (a node vector) in, psi out ordinate-major
        phr = torch.randn(ctx.n_nodes, dtype=torch.float64, device="cuda")
        t_iso64 = timed(lambda: sw.apply_iso(phr, yr, ordinate_major=True))
        t_iso32 = timed(lambda: sw.apply_iso(phr, yf, ordinate_major=True))
        apply_bytes64 = 2 * n * 8 + 2 * ctx.n_cells * 8
        apply_bytes32 = 2 * n * 4 + 2 * ctx.n_cells * 4
        sweep_bytes64 = 2 * n * 8 + ctx.n_cells * 8
        iso_bytes64 = n * 8 + ctx.n_nodes * 8 + ctx.n_cells * 8
        extra["apply_gbs"] = {"fp64": apply_bytes64 / t_apply64 / 1e6, "fp32": apply_bytes32 / t_apply32 / 1e6,
                              "fp64_us": t_apply64 * 1e3, "fp32_us": t_apply32 * 1e3}
        peak, peak_kind = _peaks()
        extra["kernels"] = kernel_map(ctx, T, prob, stream, peak, peak_kind)
        ctx.set_group(st, ss)
        extra["sweep_us"] = {"fp64": t_sweep64 * 1e3, "fp32": t_sweep32 * 1e3,
                             "fp64_iso_ordinate_major": t_iso64 * 1e3, "fp32_iso_ordinate_major": t_iso32 * 1e3}
        # Dominant kernel of the solve: one sweep per iteration; the full basis
        # adds one apply per iteration and a sweep per cycle
        compressed = stats[-1]["krylov"] == 2
        sweeps = its if compressed else its + 1
        applies = 2 if compressed else its + 1
        t_dom_sweep = t_iso64 if compressed else t_sweep64
        dom_sweep = t_dom_sweep * sweeps >= t_apply64 * applies
        peak, peak_kind = _peaks()
        # The sweep's algorithmic bytes count its matrix - each cell-ordinate's
        # B^{-1} and couplings, read from the factor store - as an SpMV's count
        # its nonzeros, beside the vectors; the vectors alone are reported too
        fac64 = sw.status()["factor_bytes_fp64"]
        bytes_counted = None
        if dom_sweep and compressed:
            # phi in (node vector), psi out, sigma_t, the factor store
            ach = (iso_bytes64 + fac64) / t_iso64 / 1e6
            ach_vec = iso_bytes64 / t_iso64 / 1e6
            kernel, traffic_key = "SweepKernel<double,3,3> (isotropic source, psi ordinate-major)", "sweep_iso_fp64"
            bytes_counted = ("psi out (N_r 8), phi in (N_n 8), sigma_t (n_c 8) and the FP64 factor store "
                             f"({fac64} B: W and the couplings of every cell-ordinate, the sweep's matrix)")
        elif dom_sweep:
            ach = (sweep_bytes64 + fac64) / t_sweep64 / 1e6
            ach_vec = sweep_bytes64 / t_sweep64 / 1e6
            kernel, traffic_key = "SweepKernel<double,3,3>", "sweep_fp64"
            bytes_counted = f"q in and psi out (2 N_r 8), sigma_t (n_c 8) and the FP64 factor store ({fac64} B)"
        else:
            ach = apply_bytes64 / t_apply64 / 1e6
            kernel, traffic_key = "ApplyKernel<double,3,3,0>", "apply_fp64"
        # DRAM bytes of one launch of that kernel, from a committed ncu capture
        # (not measured by this run)
        traffic, traffic_source = None, None
        tpath = os.path.join(ROOT, "profiles", "traffic.json")
        if os.path.exists(tpath):
            try:
                tj = json.load(open(tpath))
                traffic = tj.get(traffic_key)
                traffic_source = f"ncu capture, profiles/traffic.json [{traffic_key}]: {tj.get('_source', '')}"
            except Exception:
                traffic, traffic_source = None, None
        extra["roofline"] = {"bound": "hbm", "kernel": kernel, "achieved": ach, "peak": peak, "unit": "GB/s",
                             "frac": ach / peak, "peak_source": peak_kind, "traffic": traffic,
                             "bytes_counted": bytes_counted,
                             "achieved_vectors_only": ach_vec if dom_sweep else None,
                             "frac_vectors_only": (ach_vec / peak) if dom_sweep else None,
                             "traffic_unit": "bytes per launch", "traffic_source": traffic_source,
                             "share_of_solve": (t_dom_sweep * sweeps if dom_sweep else t_apply64 * applies) / ms}

        # ~~~ Mixed precision: FP32 operator / sweep / Krylov storage + FP64 refinement
        mixed = T.TransportSolver(ctx, rtol=1e-8, precision="mixed", pc="sweep", restart=30, max_it=500,
                                  inner_rtol=1e-5)
        xm = ctx.vector(fill=0.0)
        for _ in range(2):
            mixed.solve(b, xm)
        torch.cuda.synchronize()
        m0, m1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        m0.record(stream)
        for _ in range(args.steps):
            xm, stm = mixed.solve(b, xm)
        m1.record(stream)
        torch.cuda.synchronize()
        mixed_ms = m0.elapsed_time(m1) / args.steps
        phi64 = T.angular_integral(ctx, x)
        phim = T.angular_integral(ctx, xm)
        extra["mixed"] = {"s_per_solve": mixed_ms / 1e3, "speedup_vs_fp64": ms / mixed_ms,
                          "iterations": stm["iterations"], "outer": stm["outer"], "residual": stm["residual"],
                          "phi_rel_err_vs_fp64": float((phim - phi64).norm() / phi64.norm())}
        # The same FP64 solve with every basis vector held in full (no compressed form)
        full = T.TransportSolver(ctx, rtol=1e-8, precision="fp64", pc="sweep", restart=30, max_it=500, krylov="full")
        xf = ctx.vector(fill=0.0)
        for _ in range(2):
            full.solve(b, xf)
        torch.cuda.synchronize()
        k0, k1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        k0.record(stream)
        for _ in range(args.steps):
            xf, stf = full.solve(b, xf)
        k1.record(stream)
        torch.cuda.synchronize()
        extra["full_basis"] = {"s_per_solve": k0.elapsed_time(k1) / args.steps / 1e3, "iterations": stf["iterations"]}
        # FP64 solve back on its own workspace
        solver = T.TransportSolver(ctx, rtol=1e-8, precision="fp64", pc="sweep", restart=30, max_it=500)

        # ~~~ Adjoint gradient of the detector response over a seeded 16 x 16-cell patch
        det = torch.tensor(P.detector_patch(prob).astype(np.float64), device="cuda")
        model = T.DetectorResponse(ctx, prob.source[0], det.cpu().numpy(), rtol=1e-8, max_it=500)
        sig_t = st.clone().requires_grad_(True)
        sig_s = ss.clone().requires_grad_(True)
        for _ in range(2):
            J = model(sig_t, sig_s)
            torch.autograd.grad(J, (sig_t, sig_s))
        torch.cuda.synchronize()
        g0, g1, g2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        g0.record(stream)
        J = model(sig_t, sig_s)
        g1.record(stream)
        gt, gs = torch.autograd.grad(J, (sig_t, sig_s))
        g2.record(stream)
        torch.cuda.synchronize()
        fwd_ms, tot_ms = g0.elapsed_time(g1), g0.elapsed_time(g2)
        extra["adjoint"] = {"grad_s": tot_ms / 1e3, "forward_s": fwd_ms / 1e3,
                            "adjoint_over_forward": (tot_ms - fwd_ms) / fwd_ms,
                            "parameters": 2 * ctx.n_cells, "J": float(J.item()),
                            "adjoint_iterations": model.last_adjoint["iterations"]}
        ctx.set_group(st, ss)

    # ~~~ End to end through the public host-buffer call: every step uploads
    # its b from pinned host memory and downloads its x, on the library's two
    # copy streams, each copy overlapping a neighbouring step's solve
    hb = b.cpu().pin_memory()
    hxs = [torch.empty(n, dtype=torch.float64).pin_memory() for _ in range(2)]
    solver.solve_host_batch([hb, hb], hxs)
    torch.cuda.synchronize()
    barrier()
    torch.cuda.synchronize()
    f0, f1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    f0.record(stream)
    solver.solve_host_batch([hb] * args.steps, [hxs[i % 2] for i in range(args.steps)], stream=stream)
    f1.record(stream)
    torch.cuda.synchronize()
    e2e_ms = max_over_ranks(f0.elapsed_time(f1) / args.steps, world, "cuda")

    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cpu, xcpu = cpu_baseline(args)
        phi_c = np.asarray(T.angular_integral(ctx, x).cpu())
        import oracle as O
        phi_o = O.angular_integral(xcpu, ctx.n_nodes, q)
        cpu["phi_rel_diff_gpu_vs_cpu"] = float(np.linalg.norm(phi_c - phi_o) / np.linalg.norm(phi_o))

    ctx.close()
    # ~~~ The other solve configurations (one GPU each; under torchrun every
    # rank runs its own copy, so all ranks take the same steps)
    if not args.quick and not args.no_workloads:
        torch.cuda.empty_cache()
        extra["hex128"] = workload_hex128(args, stream)
        torch.cuda.empty_cache()
        extra["tet44"] = workload_tet44(args, stream)
        extra["cg256"] = workload_cg256(args, stream)
        extra["upscatter"] = workload_upscatter(args, stream)

    if rank == 0:
        line = {"metric": METRIC, "value": value, "unit": "s/solve", "n_gpus": world, "steps": args.steps,
                "warmup": args.warmup, "ms_per_step": ms, "higher_is_better": False, "scaling": "weak",
                "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded, PCG64 20261203+1)",
                "config": {"workload": WORKLOAD, "rows": n, "rtol": 1e-8, "iterations": its,
                           "krylov": {1: "full", 2: "compressed"}.get(stats[-1]["krylov"], "?"),
                           "true_residual": res, "preconditioner": "exact upwind sweep (patch tasks)",
                           "restart": 30, "parallelism": f"replicas{world}", "setup_s": setup_s,
                           "l2": "each step (a full solve) streams >4 GB of Krylov vectors, far above the 126 MB L2"},
                "gpu_launches": int(launches), "clocks": clk.summary(),
                "e2e": {"value": e2e_ms / 1e3, "unit": "s/solve", "h2d_bytes_per_step": n * 8,
                        "d2h_bytes_per_step": n * 8,
                        "call": "ubolt_solve_host_batch: pinned host b in, x out, copies overlapping the solves"}}
        line.update({k: v for k, v in extra.items() if k != "roofline"})
        if "roofline" in extra:
            line["roofline"] = extra["roofline"]
        if cpu:
            line["cpu_baseline"] = cpu
        print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


if __name__ == "__main__":
    main()

"""Benchmark of the femSolidmechanics Newton step on B200.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference] [--workload large|small]

A step is one full Newton iteration of the hex8 Neo-Hookean cantilever at 256(x) x 64 x 64
(1,048,576 elements, 3,257,475 DOFs), first load step (lambda = 0.2, u = 0): fused element
evaluation + scatter assembly, external loads, FP64 residual norm, Jacobi-PCG to the stated
relative tolerance (PETSc KSPCG semantics) and the displacement update. Every step starts from
the same state, so every step does identical work. The matrix (2.2 GB of FP64 values) is
larger than L2, so no flush is needed between steps.

--impl reference times the CPU restatement of the reference's path (the oracle: the
reference itself cannot be built on this image) on the host cores, on the same workload.
Under torchrun each rank runs an independent replica (the path has no exchange step).
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "Newton iters/s (hex8 Neo-Hookean cantilever 256x64x64, 3.26M DOFs, PCG to rtol 1e-8)"


def _peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def _workload(name: str):
    from mphyfem_b200 import meshgen
    if name == "small":
        return meshgen.cantilever_small()
    if name == "two_phase":
        return meshgen.two_phase_inclusions(256, 64, 64, seed=23)
    if name == "tet10":
        # 10-node tets, Kuhn split of a 96(x) x 48 x 48 grid, kappa = 100, traction 0.02, dt 0.1
        return meshgen.tet10_kuhn(96, 48, 48)
    return meshgen.cantilever_large()


def _auto_coarse(n_node: int) -> int:
    """Default size of the coarse space: about one aggregate per 1,300 nodes (24 x 6 x 6 boxes on
    the 256 x 64 x 64 hex8 cantilever, 28 x 7 x 7 on the 96 x 48 x 48 tet10 block). Larger spaces
    cut iterations but every CG iteration's GEMV reads the whole E^-1 and the dense setup grows
    with its tile count; measured sweeps on both workloads put the optimum near this density."""
    return max(8, int(round(n_node / 1300)))


def _config(prob, rtol):
    return {
        "workload": f"{prob.name}: one Newton iteration (assembly + loads + norm + PCG to true relative residual {rtol:g} "
                    f"+ update), lambda={prob.dt:g} (the first load step), u=0",
        "n_elem": prob.n_elem, "n_node": prob.n_node, "n_dof": prob.n_dof, "n_free": prob.n_free,
        "element": ("tet10, 4-point rule, near-incompressible Neo-Hookean mu=1 kappa=100 (Utype 3), jitter 0.1h seed 7"
                    if prob.npe == 10 else
                    "hex8, 2x2x2 Gauss, compressible Neo-Hookean mu=1 kappa=10 (Utype 3)" if prob.mats.shape[0] == 1
                    else "hex8, two-phase Neo-Hookean: matrix mu=1 kappa=10, spherical inclusions mu=1000 "
                         f"kappa=10000 ({prob.meta.get('stiff_elems')} elements, seed 23)"),
        "tangent": "reference (utilitiesmaterialHyperelastic.cpp as written)",
        "l2_flush": "not needed: the FP64 matrix (~2.2 GB) exceeds the 126 MB L2",
    }


class ClockSampler:
    """nvidia-smi clocks / throttle reasons sampled every 200 ms during the timed region."""

    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown," \
             "clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown," \
             "clocks_event_reasons.sw_power_cap"

    def __init__(self, device: int):
        self.device = device
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        self.out = ""
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.out, _ = self.proc.communicate(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        rows = [r.split(",") for r in (getattr(self, "out", "") or "").strip().splitlines() if r.count(",") >= 6]
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[0]) for r in rows if r[0].strip().replace(".", "").isdigit()]
        mx = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({n for r in rows for n, v in zip(names, r[3:7]) if "Active" in v and "Not" not in v})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(rows)}


def _read_traffic(kind: str):
    """DRAM bytes per launch from a committed ncu summary (a profiles/*.md line 'dram_bytes_per_launch_<kind>: X')."""
    d = os.path.join(ROOT, "profiles")
    if not os.path.isdir(d):
        return None
    key = f"dram_bytes_per_launch_{kind}:"
    for fn in sorted(os.listdir(d)):
        if fn.endswith((".txt", ".md")):
            for line in open(os.path.join(d, fn)):
                if line.strip().startswith(key):
                    try:
                        return float(line.split(":", 1)[1].split()[0])
                    except ValueError:
                        return None
    return None


# ------------------------------------------------------------------------------------- CPU side
def _threads():
    try:
        return len(os.sched_getaffinity(0))
    except Exception:
        return os.cpu_count() or 1


class CpuReference:
    """The oracle (the FP64 C++ restatement of the reference's path: element loop, Neo-Hookean,
    AIJ assembly, PETSc-KSPCG Jacobi-PCG) on the workload's own mesh and matrix, on this host's
    cores. Building it takes the reference's prepareMatrixPattern on the CPU (timed once)."""

    def __init__(self, prob):
        from oracle import binding
        binding.build()
        self.prob = prob
        self.nt = _threads()
        t0 = time.perf_counter()
        self.op = binding.OracleProblem(prob)
        self.pattern_s = time.perf_counter() - t0
        self.u0 = np.zeros(prob.n_dof)
        self.val, rhs, _, _ = self.op.assemble(self.u0, nthreads=self.nt, want_reac=False)
        self.b = rhs + prob.dt * prob.fnodal[np.flatnonzero(prob.fixed == 0)]

    def assembly_s(self, nthreads):
        t0 = time.perf_counter()
        self.op.assemble(self.u0, nthreads=nthreads, want_reac=False)
        return time.perf_counter() - t0

    def cg_iter_s(self, nthreads, its):
        """Seconds per Jacobi-PCG iteration on the workload's matrix (its iterations, no stop)."""
        t0 = time.perf_counter()
        _, done, _, _ = self.op.cg(self.val, self.b, rtol=1e-30, maxit=its, nthreads=nthreads)
        return (time.perf_counter() - t0) / max(done, 1)

    def cg_full(self, rtol, maxit):
        """Jacobi-PCG from x = 0 to ||b - A x|| <= rtol ||b|| on all cores: (its, seconds)."""
        t0 = time.perf_counter()
        _, its, _, st = self.op.cg(self.val, self.b, rtol=rtol, maxit=maxit, nthreads=self.nt, norm_type=1)
        return its, time.perf_counter() - t0, st


def cpu_baseline_sample(prob, krylov_its: int, its_source: str):
    """The CPU baseline beside the GPU numbers: one Newton iteration of the workload (assembly +
    Jacobi-PCG + update) on the oracle, timed on the workload's own data. Measured: one full
    assembly single-threaded (the reference's element loop has no OpenMP) and on all cores, and
    Jacobi-PCG iterations on the assembled matrix, 5 single-threaded and 20 on all cores. The
    iteration count to the tolerance (krylov_its, from its_source) multiplies the measured
    per-iteration time; that product is the extrapolated part. About 30-40 s of CPU work."""
    ref = CpuReference(prob)
    a1 = ref.assembly_s(1)
    an = ref.assembly_s(ref.nt)
    c1 = ref.cg_iter_s(1, 5)
    cn = ref.cg_iter_s(ref.nt, 20)
    t1 = a1 + krylov_its * c1
    tn = an + krylov_its * cn
    return {
        "value": 1.0 / tn, "unit": "Newton iter/s", "cores": ref.nt, "kind": "port",
        "sample": (f"oracle (FP64 C++ restatement of the reference path) on this workload's mesh and matrix "
                   f"({prob.n_elem} elements, {ref.op.nnz} nonzeros): one full assembly and 20 Jacobi-PCG "
                   f"iterations timed on {ref.nt} threads, x {krylov_its} Krylov iterations ({its_source})"),
        "measured": {"threads": ref.nt, "assembly_s": an, "cg_iter_s": cn, "assembly_s_1thread": a1,
                     "cg_iter_s_1thread": c1, "pattern_build_s": ref.pattern_s},
        "single_thread": {"value": 1.0 / t1, "unit": "Newton iter/s", "cores": 1},
        "krylov_its": krylov_its, "krylov_its_source": its_source,
    }


def run_reference(args):
    """The reference arm: the reference's own method (AIJ assembly + PETSc-style Jacobi-PCG, FP64)
    through the oracle on the host cores, on the same workload. Setup builds the pattern and the
    matrix and runs one complete Jacobi-PCG solve to the workload's tolerance (its iteration count
    and time are measured, not supplied). Each step is a bounded sample: one full assembly and
    10 Jacobi-PCG iterations on all cores; the step's time is that assembly plus the measured
    per-iteration time times the measured iteration count."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    prob = _workload(args.workload)
    t_setup = time.perf_counter()
    ref = CpuReference(prob)
    its, full_s, st = ref.cg_full(args.rtol, args.max_it)
    setup_s = time.perf_counter() - t_setup
    steps, walls, asm, cgi = [], [], [], []
    for k in range(max(3, args.warmup) + args.steps):
        w0 = time.perf_counter()
        a = ref.assembly_s(ref.nt)
        c = ref.cg_iter_s(ref.nt, 10)
        if k >= max(3, args.warmup):
            steps.append(a + its * c)
            asm.append(a)
            cgi.append(c)
            walls.append(time.perf_counter() - w0)
    t = statistics.median(steps)
    line = {
        "impl": "reference", "metric": METRIC, "value": 1.0 / t, "unit": "Newton iter/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": _config(prob, args.rtol),
        "method": "FP64 AIJ assembly + Jacobi-PCG (PETSc KSPCG + PCJACOBI semantics), the reference's method",
        "cpu_baseline": {
            "value": 1.0 / t, "unit": "Newton iter/s", "cores": ref.nt, "kind": "port",
            "sample": (f"oracle on the workload's own matrix ({ref.op.nnz} nonzeros): per step one full assembly "
                       f"and 10 Jacobi-PCG iterations on {ref.nt} threads; Krylov count {its} measured by one "
                       f"complete solve to the true relative residual {args.rtol:g} at setup ({full_s:.1f} s)")},
        "measured": {"threads": ref.nt, "krylov_its": its, "krylov_status": int(st), "cg_full_s": full_s,
                     "assembly_s": statistics.median(asm), "cg_iter_s": statistics.median(cgi),
                     "pattern_build_s": ref.pattern_s, "setup_s": setup_s,
                     "sample_wall_s_per_step": statistics.median(walls)},
        "e2e": {"value": 1.0 / t, "unit": "Newton iter/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
        "note": "the reference (PETSc/Eigen/Boost/MPI/VTK build) cannot be built on this image; its path is timed "
                "through the FP64 CPU restatement. ms_per_step is the full Newton iteration, from the measured "
                "assembly and per-iteration times and the measured iteration count; each step's own wall-clock "
                "is sample_wall_s_per_step",
    }
    print(json.dumps(line), flush=True)


# ------------------------------------------------------------------------------------- GPU side
def _method_name(args):
    parts = [{"fp64": "FP64", "mixed": "mixed FP32/FP64", "mixed32": "mixed FP32 vectors",
              "mixed_tc": "mixed FP32/FP64 (tensor-core split-BF16 tangent)"}[args.precision],
             {"jacobi": "Jacobi", "fsai": "FSAI", "learned": "learned FSAI"}[args.pc]]
    if args.coarse > 0:
        kind = "linear-mode" if args.coarse_modes == 12 else "rigid-body"
        parts.append(f"+ {kind} coarse space ({args.coarse} aggregates x {args.coarse_modes} modes)")
    return " ".join(parts) + "-PCG"


_GNN = []


def _make_solver(api, _lib, mesh, pat, args, precision, pc, coarse):
    sol = api.SolverGpu(mesh, pat, rtol=args.rtol, max_it=args.max_it,
                        precision={"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED,
                                   "mixed32": _lib.PREC_MIXED_F32VEC, "mixed_tc": _lib.PREC_MIXED_TC}[precision],
                        pc_type={"jacobi": _lib.PC_JACOBI, "fsai": _lib.PC_FSAI,
                                 "learned": _lib.PC_FSAI_LEARNED}[pc],
                        inner_rtol=args.inner_rtol, max_outer=args.max_outer, coarse_aggregates=coarse,
                        coarse_modes=args.coarse_modes,
                        norm_type=args.norm)
    if pc == "learned":
        from mphyfem_b200 import learned
        if not _GNN:
            _GNN.append(learned.Gnn(mesh.ctx, learned.load_params(args.gnn or learned.DEFAULT_WEIGHTS)))
        _GNN[0].attach(sol)
    return sol


def _time_steps(torch, stream, step, steps, warmup):
    for _ in range(warmup):
        step()
    torch.cuda.synchronize()
    ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    stats = []
    ev0.record(stream)
    for _ in range(steps):
        stats.append(step())
    ev1.record(stream)
    torch.cuda.synchronize()
    return ev0.elapsed_time(ev1), stats


def _time_leg(torch, api, _lib, mesh, pat, args, prob, disp, fext, dev, method, steps):
    """One more method on the bench step (u = 0, lambda = dt, one Newton iteration): one untimed
    iteration (graphs, preconditioner buffers), then `steps` timed with events on its stream."""
    precision, pc, coarse = method
    s = _make_solver(api, _lib, mesh, pat, args, precision, pc, coarse)
    st = torch.cuda.ExternalStream(s.stream, device=dev)

    def step():
        disp.zero_()
        return s.newton_iteration(disp, fext, prob.dt)

    t, stats = _time_steps(torch, st, step, steps, 1)
    out = {"method": _method_name(argparse.Namespace(**dict(vars(args), precision=precision, pc=pc, coarse=coarse))),
           "ms_per_newton_iter": t / len(stats),
           "krylov_its": int(statistics.median([q.krylov_its for q in stats])),
           "krylov_status": sorted({_lib.status_string(int(q.status)) for q in stats}),
           "true_relres": s.true_residual(),
           "solve_ms": statistics.median([q.t_solve_ms for q in stats]),
           "assembly_ms": statistics.median([q.t_assembly_ms for q in stats])}
    if pc != "jacobi":
        pcl = s.pc_last()
        out["preconditioner"] = {"setup_ms": pcl["setup_ms"], "fallback": pcl["fallback"],
                                 "first_relres": pcl["first_relres"]}
    if coarse > 0:
        out["coarse_setup_ms"] = s.coarse_info()["setup_ms"]
    s.close()
    return out


def _other_workloads(torch, api, _lib, args, dev):
    """The two other GPU workloads of the north star, measured in the default run so that their
    figures come from the same run as the headline (each after the headline's buffers are freed):
      - tet10: the 10-node-tet Kuhn cantilever 96(x) x 48 x 48 (1.33 M elements, 5.45 M DOFs),
        near-incompressible (kappa = 100), the headline's method, one Newton iteration from u = 0
        (one untimed, two timed);
      - batched: 512 independent hex8 blocks (batched_blocks(512, seed=11), 2.09 M elements,
        7.79 M DOFs), FP64, consistent tangent, persistent cluster PCG with 8 rigid-body slabs per
        instance on the (2 CTAs, 512 threads) schedule, every instance's 5 load steps with Newton
        to 1e-8 and PCG to true residual 1e-10: one whole job, timed by the library's events."""
    from mphyfem_b200 import meshgen, ranks
    out = {}
    q = meshgen.tet10_kuhn(96, 48, 48)
    mesh = api.Mesh(api.Context(0), q)
    pat = api.Pattern(mesh)
    disp = torch.zeros(q.n_dof, dtype=torch.float64, device=dev)
    fext = torch.tensor(q.fnodal, device=dev)
    coarse = _auto_coarse(q.n_node) if getattr(args, "coarse_auto", False) else args.coarse
    leg = _time_leg(torch, api, _lib, mesh, pat, args, q, disp, fext, dev, (args.precision, args.pc, coarse), 2)
    leg.update({"workload": f"{q.name}: {q.n_elem} tet10 elements, {q.n_dof} DOFs, one Newton iteration from u = 0 at "
                            f"lambda = {q.dt:g}, PCG to true relative residual {args.rtol:g}",
                "melems_per_s_assembly": q.n_elem / (leg["assembly_ms"] * 1e-3) / 1e6})
    out["tet10_gpu"] = leg
    del mesh, pat, disp, fext
    allp = meshgen.batched_blocks(512, seed=11)
    for b in allp:
        b.newton_rtol = 1e-8
    ctx = api.Context(0)
    _, bat = ranks.batched_share(allp, 0, 1, ctx, schedule=(2, 512), coarse_slabs=8, precision=_lib.PREC_FP64,
                                 rtol=1e-10, norm_type=1, max_it=args.max_it, tangent=_lib.TANGENT_CONSISTENT)
    o = bat.newton_run(max_newton=15)
    out["batched_gpu"] = {
        "workload": "batched_blocks(512, seed=11): 512 hex8 blocks, nx, ny ~ U{4..16}, nz ~ U{16..64}, 5 load steps "
                    "each, Newton to 1e-8, PCG to true relative residual 1e-10, FP64, 8 rigid-body slabs",
        "n_elem": sum(b.n_elem for b in allp), "n_dof": sum(b.n_dof for b in allp),
        "ms_per_job": o["stats"]["t_ms"], "instances_per_s": len(allp) / (o["stats"]["t_ms"] * 1e-3),
        "graph_replays": o["stats"]["graph_replays"], "kernel_launches": o["stats"]["kernel_launches"],
        "krylov_its_mean": float(o["krylov_its"].mean()), "cuts": int(o["cuts"].sum()),
        "instances_ok": int((o["status"] == 0).sum()), "schedule": list(bat.schedule())}
    bat.close()
    return out


def _parity_first_step(api, _lib, mesh, pat, args, prob, legs, newton_rtol=1e-8, max_newton=15):
    """Accuracy at the workload's size: the first load step (lambda = dt from u = 0) converged to
    ||R|| < newton_rtol ||R_first|| with the consistent tangent (the reference's tangent need not
    converge quadratically, or at all, at this load), by the plain FP64 GPU method (FP64 element
    kernel, FP64 matrix, FP64 Jacobi-PCG: the FP64 solution) and by each method of `legs`.
    Reports every method's Newton history and max|u - u64| / max|u64|. max_newton leaves room
    for the FP32 tangent's slower final Newton iterations (its Jacobian is accurate to about
    1e-7), which the histories show."""
    def run(method):
        precision, pc, coarse = method
        a = argparse.Namespace(**dict(vars(args), precision=precision, pc=pc, coarse=coarse))
        s = api.SolverGpu(mesh, pat, rtol=args.rtol, max_it=args.max_it,
                          precision={"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED,
                                     "mixed32": _lib.PREC_MIXED_F32VEC, "mixed_tc": _lib.PREC_MIXED_TC}[precision],
                          pc_type={"jacobi": _lib.PC_JACOBI, "fsai": _lib.PC_FSAI,
                                   "learned": _lib.PC_FSAI_LEARNED}[pc],
                          inner_rtol=args.inner_rtol, max_outer=args.max_outer, coarse_aggregates=coarse,
                          coarse_modes=args.coarse_modes, norm_type=args.norm, tangent=_lib.TANGENT_CONSISTENT)
        if pc == "learned":
            _GNN[0].attach(s)
        t0 = time.perf_counter()
        r = api.newton_run(s, prob, max_newton=max_newton, tol_rel=newton_rtol, t_final=prob.dt, max_steps=1)
        wall = time.perf_counter() - t0
        s.close()
        hist = [{"iter": int(h[1]), "rhs_norm": float(h[2]), "krylov_its": int(h[3]),
                 "krylov_status": _lib.status_string(int(h[4]))} for h in r.hist]
        # a try that does not converge is cut (MyTime::cut: dt halved, the step retried from the
        # last converged state): every try starts at iteration 1
        tries = np.flatnonzero(r.hist[:, 1] == 1) if len(r.hist) else np.array([0])
        cuts = max(0, len(tries) - 1)
        last = r.hist[tries[-1]:] if len(r.hist) else r.hist
        conv = cuts == 0 and len(last) > 0 and last[-1, 2] < newton_rtol * last[0, 2]
        return r.disp, {"method": _method_name(a), "newton": hist, "converged": bool(conv), "cuts": cuts,
                        "lambda_reached": prob.dt / 2 ** cuts,
                        "newton_status": _lib.status_string(int(r.status)), "wall_s": wall}

    u64, ref = run(("fp64", "jacobi", 0))
    out = {"case": f"first load step (lambda={prob.dt:g}) from u=0 to ||R|| < {newton_rtol:g} ||R_first||, "
                   f"consistent tangent, Krylov to true relative residual {args.rtol:g}, at most {max_newton} "
                   f"Newton iterations",
           "fp64": ref}
    scale = float(np.abs(u64).max())
    for name, m in legs.items():
        u, rec = run(m)
        rec["disp_err_vs_fp64"] = float(np.abs(u - u64).max() / scale)
        out[name] = rec
    out["max_abs_u_fp64"] = scale
    return out


def run_ours(args):
    import torch
    import torch.distributed as dist

    from mphyfem_b200 import ranks
    rank, local, world = ranks.world_info()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=600))
    if not torch.cuda.is_available():
        print(json.dumps({"metric": METRIC, "error": "no CUDA device"}))
        sys.exit(2)
    from mphyfem_b200 import _lib, api

    dev = f"cuda:{local}"
    prob = _workload(args.workload)
    args.coarse_auto = args.coarse < 0
    if args.coarse_auto:
        args.coarse = _auto_coarse(prob.n_node)
    ctx = api.Context(local)
    mesh = api.Mesh(ctx, prob)
    pat = api.Pattern(mesh)
    sol = _make_solver(api, _lib, mesh, pat, args, args.precision, args.pc, args.coarse)
    stream = torch.cuda.ExternalStream(sol.stream, device=dev)
    disp = torch.zeros(prob.n_dof, dtype=torch.float64, device=dev)
    fext = torch.tensor(prob.fnodal, dtype=torch.float64, device=dev)

    def step():
        disp.zero_()
        return sol.newton_iteration(disp, fext, prob.dt)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    with ClockSampler(local) as clk:
        ms, stats = _time_steps(torch, stream, step, args.steps, 0)
    if world > 1:
        dist.barrier()
    ms = ranks.max_over_ranks(ms, dev)  # the job's time is its slowest rank's
    its = [s.krylov_its for s in stats]
    kstatus = sorted({int(s.status) for s in stats})
    asm_ms = statistics.median([s.t_assembly_ms for s in stats])
    solve_ms = statistics.median([s.t_solve_ms for s in stats])
    launches = int(sum(s.kernel_launches for s in stats))
    relres = sol.true_residual()
    coarse = sol.coarse_info() if args.coarse > 0 else None
    pc_info = sol.pc_last() if args.pc != "jacobi" else None

    # dominant kernel: the SpMV of the Krylov loop (the same kernel: y = A p with the fused p.Ap),
    # timed back to back with events on its stream; each call also zeroes its 96-byte state
    mi = sol.matrix_info()
    x = torch.randn(prob.n_dof, dtype=torch.float64, device=dev)
    y = torch.empty_like(x)
    for _ in range(3):
        sol.spmv_dot(x, y, want_dot=False)
    nrep = 20
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(nrep):
        sol.spmv_dot(x, y, want_dot=False)
    e1.record(stream)
    torch.cuda.synchronize()
    spmv_ms = e0.elapsed_time(e1) / nrep
    vbytes = mi["value_bytes"] // (9 * mi["stored_blocks"])  # 8 (FP64) or 4 (FP32) per value
    if vbytes == 8:
        spmv_bytes = mi["true_blocks"] * (9 * 8 + 4) + 2 * prob.n_dof * 8
    else:
        # the FP32 storage holds the off-diagonal blocks only (each row's diagonal block is formed
        # from them in the kernel), plus the prescribed-DOF mask
        spmv_bytes = (mi["true_blocks"] - prob.n_node) * (9 * 4 + 4) + 2 * prob.n_dof * 8 + prob.n_node * 3
    peak, peak_kind = _peaks()
    achieved = spmv_bytes / (spmv_ms * 1e-3) / 1e9
    # assembly: each matrix value written once (FP32: off-diagonal blocks plus the FP64 Jacobi
    # diagonal), the residual, coordinates and displacements read, the connectivity read
    if vbytes == 8:
        mat_bytes = pat.nnz * 8
    else:
        mat_bytes = (pat.nnz - 9 * prob.n_node) * 4 + prob.n_dof * 8
    asm_bytes = mat_bytes + prob.n_free * 8 + prob.n_node * 48 + prob.n_elem * 36

    # end to end through the C ABI with host buffers (H2D of u and f_ext, D2H of u every step)
    disp_h = torch.zeros(prob.n_dof, dtype=torch.float64).pin_memory().numpy()
    fext_h = torch.tensor(prob.fnodal, dtype=torch.float64).pin_memory().numpy()
    e2e_steps = max(1, min(args.steps, 3))
    sol.newton_iteration_host(disp_h, fext_h, prob.dt)
    e2e_total = 0.0
    for _ in range(e2e_steps):
        # back to u = 0 so that every step is the same Newton iteration: a reset of the
        # harness's buffer, outside the timed call
        disp_h[:] = 0.0
        e0.record(stream)
        sol.newton_iteration_host(disp_h, fext_h, prob.dt)  # returns after its D2H copy
        e1.record(stream)
        e1.synchronize()
        e2e_total += e0.elapsed_time(e1)
    e2e_ms = ranks.max_over_ranks(e2e_total / e2e_steps, dev)

    # the other methods on the same workload and step, measured in the same run (1 GPU): the
    # plain GPU method (FP64 Jacobi-PCG, the drop-in for the reference's KSPCG + PCJACOBI) and the
    # learned factorised preconditioner with the same coarse space
    plain = learned_leg = parity = others = None
    headline = (args.precision, args.pc, args.coarse)
    if world == 1:
        sol.close()
        if not args.no_plain and headline != ("fp64", "jacobi", 0):
            plain = _time_leg(torch, api, _lib, mesh, pat, args, prob, disp, fext, dev, ("fp64", "jacobi", 0),
                              max(1, min(args.steps, 2)))
            plain["speedup_of_this_method"] = plain["ms_per_newton_iter"] / (ms / args.steps)
        if not args.no_learned and headline[1] != "learned":
            lh = (args.precision, "learned", args.coarse)
            learned_leg = _time_leg(torch, api, _lib, mesh, pat, args, prob, disp, fext, dev, lh,
                                    max(1, min(args.steps, 3)))
            learned_leg["ms_vs_headline"] = learned_leg["ms_per_newton_iter"] / (ms / args.steps)
        if not args.no_parity:
            legs = {"headline": headline}
            if learned_leg is not None:
                legs["learned"] = (args.precision, "learned", args.coarse)
            parity = _parity_first_step(api, _lib, mesh, pat, args, prob, legs)
            if learned_leg is not None:
                learned_leg["disp_err_vs_fp64"] = parity["learned"]["disp_err_vs_fp64"]
        if not args.no_others and args.workload == "large":
            others = _other_workloads(torch, api, _lib, args, dev)

    if rank != 0:
        if world > 1:
            dist.destroy_process_group()
        return
    cpu = None
    if world == 1 and not args.no_cpu:
        if plain is not None:
            k_its, k_src = plain["krylov_its"], "the Jacobi-PCG count of the plain FP64 GPU leg measured in this run"
        else:
            k_its, k_src = int(statistics.median(its)), "this run's Krylov count"
        cpu = cpu_baseline_sample(prob, k_its, k_src)
    line = {
        "metric": METRIC, "value": world * args.steps / (ms * 1e-3), "unit": "Newton iter/s", "n_gpus": world,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32+f64",
        "data": "synthetic",
        "config": _config(prob, args.rtol),
        "method": _method_name(args),
        "parallelism": f"replicas{world}" if world > 1 else "single",
        "krylov_its": int(statistics.median(its)),
        "krylov_status": [_lib.status_string(k) for k in kstatus],
        "true_relres": relres,
        "solve_ms": solve_ms,
        "coarse": coarse,
        "preconditioner_setup": pc_info,
        "assembly": {"ms": asm_ms, "melems_per_s": prob.n_elem / (asm_ms * 1e-3) / 1e6,
                     "algorithmic_bytes": asm_bytes, "achieved_gbs": asm_bytes / (asm_ms * 1e-3) / 1e9,
                     "frac": asm_bytes / (asm_ms * 1e-3) / 1e9 / peak},
        "plain_gpu": plain,
        "learned_gpu": learned_leg,
        "other_workloads": others,
        "parity": parity,
        "e2e": {"value": world * 1e3 / e2e_ms, "unit": "Newton iter/s", "h2d_bytes_per_step": 2 * prob.n_dof * 8,
                "d2h_bytes_per_step": prob.n_dof * 8},
        "roofline": {"kernel": f"spmv_kernel with p.Ap, as in the CG iteration (SELL-32 3x3, "
                               f"{'FP64' if vbytes == 8 else 'FP32 off-diagonal'} values, FP64 vectors)",
                     "bound": "hbm", "achieved": achieved, "peak": peak, "peak_source": peak_kind, "unit": "GB/s",
                     "frac": achieved / peak,
                     "traffic": _read_traffic("spmv_fp64" if vbytes == 8 else "spmv_mixed"),
                     "algorithmic_bytes": spmv_bytes, "launch_ms": spmv_ms},
        "cpu_baseline": None if cpu is None else {k: cpu[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                                      "measured", "single_thread", "krylov_its")},
        "clocks": clk.summary(),
        "gpu_launches": launches,
    }
    print(json.dumps(line), flush=True)
    if world > 1:
        dist.destroy_process_group()


def run_batched(args):
    """The batched form: 512 independent hex8 blocks (seed 11), every instance's 5 load steps.
    One step = the whole job of this rank's share of the instances (LPT by element count), so
    run it with --steps 1 --warmup 1. Ranks share nothing on the data path; the job's time is the
    slowest rank's and the value counts every rank's instances."""
    import torch
    import torch.distributed as dist
    from mphyfem_b200 import _lib, api, meshgen, ranks
    rank, local, world = ranks.world_info()
    if world > 1:
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=__import__("datetime").timedelta(seconds=900))
    dev = f"cuda:{local}"
    allp = meshgen.batched_blocks(512, seed=11)
    for q in allp:
        q.newton_rtol = 1e-8
    ctx = api.Context(local)
    prec = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED}.get(args.precision, _lib.PREC_MIXED)
    mine, b = ranks.batched_share(allp, rank, world, ctx, coarse_slabs=8 if args.coarse != 0 else 0, precision=prec,
                                  rtol=1e-10, norm_type=1, max_it=args.max_it, tangent=_lib.TANGENT_CONSISTENT)
    probs = [allp[i] for i in mine]
    for _ in range(args.warmup):
        b.newton_run(max_newton=15)
    torch.cuda.synchronize()
    if world > 1:
        dist.barrier()
    outs = []
    with ClockSampler(local) as clk:
        for _ in range(args.steps):
            outs.append(b.newton_run(max_newton=15))
    ms = ranks.max_over_ranks(sum(o["stats"]["t_ms"] for o in outs), dev)
    total = len(allp)
    if rank == 0:
        o = outs[-1]
        print(json.dumps({
            "metric": "instances/s (512 batched hex8 Neo-Hookean blocks, 5 load steps each, Newton to 1e-8)",
            "value": total * args.steps / (ms * 1e-3), "unit": "instances/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
            "scaling": "strong", "vs_baseline": None, "dtype": "f64" if prec == _lib.PREC_FP64 else "f32+f64",
            "data": "synthetic",
            "config": {"workload": "batched_blocks(512, seed=11): nx, ny ~ U{4..16}, nz ~ U{16..64}, mu, nu, |t| "
                                   "per instance; consistent tangent; PCG to true relative residual 1e-10",
                       "n_elem": sum(q.n_elem for q in allp), "instances_rank0": len(probs),
                       "method": "persistent cluster PCG" + (" + 8 rigid-body slabs" if args.coarse != 0 else ""),
                       "schedule_rank0": list(b.schedule()),
                       "parallelism": f"instances sharded over {world} ranks" if world > 1 else "single"},
            "graph_replays_rank0": o["stats"]["graph_replays"], "kernel_launches_rank0": o["stats"]["kernel_launches"],
            "krylov_its_mean_rank0": float(o["krylov_its"].mean()), "cuts_rank0": int(o["cuts"].sum()),
            "instances_ok_rank0": int((o["status"] == 0).sum()),
            "clocks": clk.summary(), "gpu_launches": int(sum(q["stats"]["kernel_launches"] for q in outs)),
        }), flush=True)
    b.close()
    if world > 1:
        dist.destroy_process_group()


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="large", choices=["large", "small", "two_phase", "tet10", "batched"])
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--precision", default="mixed", choices=["fp64", "mixed", "mixed32", "mixed_tc"])
    ap.add_argument("--inner-rtol", dest="inner_rtol", type=float, default=0.0)
    ap.add_argument("--max-outer", dest="max_outer", type=int, default=4)
    ap.add_argument("--pc", default="jacobi", choices=["jacobi", "fsai", "learned"])
    ap.add_argument("--gnn", default=None, help="weights of the learned FSAI (default: the packaged ones)")
    ap.add_argument("--norm", type=int, default=1, choices=[0, 1],
                    help="Krylov stopping norm: 1 = true residual ||b - Ax|| <= rtol ||b|| (every method compared "
                         "at the same accuracy), 0 = PETSc's preconditioned-residual default")
    ap.add_argument("--coarse", type=int, default=-1,
                    help="aggregates of the two-level coarse correction (0: off; -1: about one per 1,300 nodes, "
                         "which gives the 24 x 6 x 6 grid at the headline size)")
    ap.add_argument("--coarse-modes", dest="coarse_modes", type=int, default=6, choices=[6, 12],
                    help="modes per aggregate: 6 rigid-body, 12 linear displacement")
    ap.add_argument("--no-plain", dest="no_plain", action="store_true",
                    help="skip the same-run measurement of the plain FP64 Jacobi-PCG method")
    ap.add_argument("--max-it", dest="max_it", type=int, default=20000)
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--no-learned", dest="no_learned", action="store_true",
                    help="skip the same-run measurement of the learned factorised preconditioner")
    ap.add_argument("--no-parity", dest="no_parity", action="store_true",
                    help="skip the first-load-step accuracy check against the FP64 GPU solution")
    ap.add_argument("--no-others", dest="no_others", action="store_true",
                    help="skip the tet10 and batched workloads measured after the headline")
    args = ap.parse_args()
    if args.impl == "reference" and args.workload == "batched":
        if int(os.environ.get("RANK", "0")) == 0:
            print(json.dumps({"impl": "reference", "unavailable": "the batched form has no single reference run; "
                              "the CPU restatement solves one instance per call (see --workload large)"}))
    elif args.impl == "reference":
        run_reference(args)
    elif args.workload == "batched":
        run_batched(args)
    else:
        run_ours(args)


if __name__ == "__main__":
    main()

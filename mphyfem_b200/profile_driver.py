"""Small, self-terminating workloads for ncu captures of single kernels.

    python -m mphyfem_b200.profile_driver --op spmv --nx 128 --ny 32 --nz 32 --reps 4
    python -m mphyfem_b200.profile_driver --op spmv --precision mixed --reps 4
    python -m mphyfem_b200.profile_driver --op assemble --nx 128 --ny 32 --nz 32 --reps 3
    python -m mphyfem_b200.profile_driver --op assemble --precision mixed_tc --reps 3
    python -m mphyfem_b200.profile_driver --op newton --precision mixed --coarse 64 --reps 1
    python -m mphyfem_b200.profile_driver --op batch --instances 48 --reps 2
    python -m mphyfem_b200.profile_driver --op assemble --model 2 --reps 3
    python -m mphyfem_b200.profile_driver --op mixed --nx 48 --ny 24 --nz 24 --reps 1

Each run builds the hex8 cantilever of the given size (or, for ``batch``, the first blocks of
the 512-block batched set), assembles it once at u = 0 and then repeats the chosen operation:
SpMV with the assembled matrix, the fused assembly, one Newton iteration (assembly + PCG +
update), or the batched persistent solve of all instances. ``--model`` gives every element one
hyperelastic model (1 Mooney-Rivlin, 2 Gent, 3 Arruda-Boyce: the dense-tangent element kernel).
The mean device time per repetition (CUDA events on the library's stream) goes to stderr.
``mixed`` builds the tet10 Kuhn mesh of the given size as a mixed u-p problem (linear vertex
pressure, kappa/mu = 1e4) and runs one load step of its Newton driver, printing per iteration
the assembly and MINRES times and iterations.
"""
from __future__ import annotations

import argparse
import sys

import numpy as np


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--op", choices=["spmv", "assemble", "newton", "batch", "mixed"], default="spmv")
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--ny", type=int, default=32)
    ap.add_argument("--nz", type=int, default=32)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--rtol", type=float, default=1e-8)
    ap.add_argument("--precision", choices=["fp64", "mixed", "mixed_tc"], default="fp64")
    ap.add_argument("--pc", choices=["jacobi", "fsai"], default="jacobi")
    ap.add_argument("--coarse", type=int, default=0)
    ap.add_argument("--instances", type=int, default=48)
    ap.add_argument("--cluster", type=int, default=4)
    ap.add_argument("--threads", type=int, default=512)
    ap.add_argument("--model", type=int, default=0, choices=[0, 1, 2, 3])
    args = ap.parse_args(argv)

    import torch

    from . import _lib, api, meshgen
    prec = {"fp64": _lib.PREC_FP64, "mixed": _lib.PREC_MIXED, "mixed_tc": _lib.PREC_MIXED_TC}[args.precision]
    ctx = api.Context(0)
    if args.op == "batch":
        probs = meshgen.batched_blocks(512, seed=11)[:args.instances]
        b = api.BatchGpu(probs, ctx, precision=prec, rtol=args.rtol, norm_type=1, max_it=20000)
        u = b.union
        b.solver.calcStiffnessAndResidual(torch.zeros(u.n_dof, dtype=torch.float64, device="cuda"))
        b.solver.addExternalForces(torch.tensor(u.fnodal, device="cuda"), 0.2)
        b.set_schedule(args.cluster, args.threads)
        for _ in range(args.reps):
            its, st, _, ms = b.solve()
        torch.cuda.synchronize()
        print(f"batch of {args.instances}: n_node={u.n_node} its mean {its.mean():.0f} max {its.max()} "
              f"ms {ms:.2f}", file=sys.stderr)
        return
    if args.op == "mixed":
        q = meshgen.tet10_kuhn(args.nx, args.ny, args.nz, lx=4.0, traction=(0.0, 0.0, -0.02), kappa=1.0e4)
        q.dt, q.t_final, q.max_steps, q.newton_rtol = 0.2, 0.2, 1, 1e-8
        m = api.MixedSolidGpu(q, ctx, tangent=_lib.TANGENT_CONSISTENT, rtol=args.rtol, max_it=200000,
                              coarse_aggregates=args.coarse)
        for _ in range(args.reps):
            res = m.solveWithNewtonRaphson(max_newton=10)
            for row in res.hist:
                print(f"iter {int(row[1])}: |R| {row[2]:.3e} minres_its {int(row[3])} "
                      f"assembly_ms {row[5]:.2f} solve_ms {row[6]:.1f}", file=sys.stderr)
        print(f"{q.name}: n_dof={q.n_dof} n_pres={m.n_pres} n_elem={q.n_elem} coupling_entries={m.nnz_coupling}")
        return
    p = meshgen.hex8_cantilever(args.nx, args.ny, args.nz)
    if args.model:
        p.mat_model = np.array([args.model], np.int32)
        p.mat_data = np.array([{1: [0.5, 0.1, 0, 0], 2: [1.0, 12.0, 0, 0], 3: [1.0, 5.0, 0, 0]}[args.model]])
        p.mats[0, 0] = p.mat_data[0, 0]
    mesh = api.Mesh(ctx, p)
    pat = api.Pattern(mesh)
    sol = api.SolverGpu(mesh, pat, rtol=args.rtol, max_it=20000, precision=prec,
                        pc_type={"jacobi": _lib.PC_JACOBI, "fsai": _lib.PC_FSAI}[args.pc],
                        coarse_aggregates=args.coarse, norm_type=1)
    disp = torch.zeros(p.n_dof, dtype=torch.float64, device="cuda")
    fext = torch.tensor(p.fnodal, dtype=torch.float64, device="cuda")
    sol.calcStiffnessAndResidual(disp)
    x = torch.randn(p.n_dof, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    stream = torch.cuda.ExternalStream(sol.stream)
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    torch.cuda.synchronize()
    e0.record(stream)
    for _ in range(args.reps):
        if args.op == "spmv":
            sol.spmv(x, y)
        elif args.op == "assemble":
            sol.calcStiffnessAndResidual(disp)
        else:
            disp.zero_()
            st = sol.newton_iteration(disp, fext, 0.2)
            print(f"krylov_its={st.krylov_its}", file=sys.stderr)
    e1.record(stream)
    torch.cuda.synchronize()
    print(f"{args.op}: {e0.elapsed_time(e1) / max(1, args.reps):.3f} ms per repetition", file=sys.stderr)
    mi = sol.matrix_info()
    print(f"{p.name}: n_dof={p.n_dof} nnz={pat.nnz} blocks={mi['true_blocks']} stored={mi['stored_blocks']} "
          f"value_bytes={mi['value_bytes']}")


if __name__ == "__main__":
    main()

"""Small, self-terminating workloads for ncu captures of single kernels.

    python -m mphyfem_b200.profile_driver --op spmv --nx 128 --ny 32 --nz 32 --reps 4
    python -m mphyfem_b200.profile_driver --op assemble --nx 128 --ny 32 --nz 32 --reps 3
    python -m mphyfem_b200.profile_driver --op newton --nx 128 --ny 32 --nz 32 --reps 1

Each run builds the hex8 cantilever of the given size, assembles it once at u = 0 and then
repeats the chosen operation: SpMV with the assembled matrix, the fused assembly, or one Newton
iteration (assembly + Jacobi-PCG + update).
"""
from __future__ import annotations

import argparse
import sys


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--op", choices=["spmv", "assemble", "newton"], default="spmv")
    ap.add_argument("--nx", type=int, default=128)
    ap.add_argument("--ny", type=int, default=32)
    ap.add_argument("--nz", type=int, default=32)
    ap.add_argument("--reps", type=int, default=3)
    ap.add_argument("--rtol", type=float, default=1e-8)
    args = ap.parse_args(argv)

    import torch

    from . import api, meshgen
    p = meshgen.hex8_cantilever(args.nx, args.ny, args.nz)
    ctx = api.Context(0)
    mesh = api.Mesh(ctx, p)
    pat = api.Pattern(mesh)
    sol = api.SolverGpu(mesh, pat, rtol=args.rtol, max_it=20000)
    disp = torch.zeros(p.n_dof, dtype=torch.float64, device="cuda")
    fext = torch.tensor(p.fnodal, dtype=torch.float64, device="cuda")
    sol.calcStiffnessAndResidual(disp)
    x = torch.randn(p.n_dof, dtype=torch.float64, device="cuda")
    y = torch.empty_like(x)
    for _ in range(args.reps):
        if args.op == "spmv":
            sol.spmv(x, y)
        elif args.op == "assemble":
            sol.calcStiffnessAndResidual(disp)
        else:
            disp.zero_()
            st = sol.newton_iteration(disp, fext, 0.2)
            print(f"krylov_its={st.krylov_its}", file=sys.stderr)
    torch.cuda.synchronize()
    mi = sol.matrix_info()
    print(f"{p.name}: n_dof={p.n_dof} nnz={pat.nnz} blocks={mi['true_blocks']} stored={mi['stored_blocks']} "
          f"value_bytes={mi['value_bytes']}")


if __name__ == "__main__":
    main()

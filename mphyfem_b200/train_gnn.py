"""Training of the learned FSAI network on data the method itself produces.

    python -m mphyfem_b200.train_gnn [--out mphyfem_b200/data/fsai_gnn.npz] [--dump DIR]

Data:
  * the batched form: the first ``n_batch`` blocks of the 512-block set (seed 11) are solved to
    convergence by the batched driver (5 load steps, consistent tangent); the tangent operators at
    the converged states are training operators, and ``--dump`` saves them with the solutions;
  * seeded two-phase inclusion layouts (spheres of radius U(0.03, 0.08), mu ratio 1000,
    kappa/mu = 10, 20 % volume fraction) at 128x32x32, each assembled at u = 0.
Every step is one Adam step of the library's own forward/backward kernels against the exact
block FSAI of the operator (mphy_gnn_train_step). Layouts are generated, used and released one
at a time, so the device holds one layout's operator at a time.
"""
from __future__ import annotations

import argparse
import math
import os
import time

import numpy as np

from . import _lib as L
from . import api, learned, meshgen


def batched_training_data(ctx, n_batch: int = 64, dump: str | None = None, log=print):
    """Solves the first n_batch blocks of the batched form; returns (union problem, converged
    displacements). With dump, writes the instances' tangents (free-DOF CSR, FP32 values) and
    solutions to dump/batched_tangents.npz."""
    import torch
    probs = meshgen.batched_blocks(512, seed=11)[:n_batch]
    for q in probs:
        q.newton_rtol = 1e-8
    b = api.BatchGpu(probs, ctx, rtol=1e-10, norm_type=1, tangent=L.TANGENT_CONSISTENT, max_it=20000)
    t0 = time.time()
    out = b.newton_run(max_newton=15)
    log(f"batched data: {n_batch} instances solved in {time.time() - t0:.1f} s, "
        f"status {np.unique(out['status']).tolist()}, cuts {int(out['cuts'].sum())}")
    union, disp = b.union, out["disp"]
    if dump:
        os.makedirs(dump, exist_ok=True)
        sol = b.solver
        sol.calcStiffnessAndResidual(torch.tensor(disp, device="cuda"))
        val, rhs, _ = sol.export(want_reac=False)
        rp, col = b.pattern.export_csr()
        assy, _ = b.pattern.export_dofmap()
        np.savez_compressed(os.path.join(dump, "batched_tangents.npz"), rowptr=rp, col=col,
                            val=val.astype(np.float32), rhs=rhs, assy=assy, disp=disp,
                            inst_node_ptr=b.node_ptr, status=out["status"])
    b.close()
    return union, disp


def _assembled(ctx, prob, disp=None):
    import torch
    mesh = api.Mesh(ctx, prob)
    pat = api.Pattern(mesh)
    sol = api.SolverGpu(mesh, pat, pc_type=L.PC_FSAI_LEARNED, precision=L.PREC_MIXED,
                        tangent=L.TANGENT_CONSISTENT)
    u = np.zeros(prob.n_dof) if disp is None else disp
    sol.calcStiffnessAndResidual(torch.tensor(u, dtype=torch.float64, device="cuda"))
    return mesh, pat, sol


def train_default(ctx, n_layouts: int = 200, size=(128, 32, 32), n_batch: int = 64, epochs: int = 3,
                  steps_per_layout: int = 4, lr: float = 2e-3, seed: int = 0, dump: str | None = None, log=print):
    """Returns (network, losses). The learning rate follows a cosine from lr to lr / 10."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gnn = learned.Gnn(ctx, seed=seed)
    union, disp = batched_training_data(ctx, n_batch, dump, log)
    bmesh, bpat, bsol = _assembled(ctx, union, disp)
    nx, ny, nz = size
    total = epochs * n_layouts * steps_per_layout
    losses, k = [], 0
    t0 = time.time()
    for ep in range(epochs):
        for j, i in enumerate(rng.permutation(n_layouts)):
            prob = meshgen.two_phase_inclusions(nx, ny, nz, seed=1000 + int(i))
            mesh, pat, sol = _assembled(ctx, prob)
            for _ in range(steps_per_layout):
                cur = lr * (0.1 + 0.9 * 0.5 * (1.0 + math.cos(math.pi * k / total)))
                losses.append(gnn.train_step(sol, cur))
                k += 1
            sol.close()
            pat.close()
            mesh.close()
            if j % 8 == 0:
                losses.append(gnn.train_step(bsol, lr * 0.5))
            if j % 25 == 0:
                log(f"epoch {ep} layout {j}: loss {np.mean(losses[-8:]):.4e} ({time.time() - t0:.0f} s)")
    bsol.close()
    return gnn, np.array(losses)


def main():
    ap = argparse.ArgumentParser(description=__doc__.splitlines()[0])
    ap.add_argument("--out", default=learned.DEFAULT_WEIGHTS)
    ap.add_argument("--dump", default=None, help="directory for the batched form's tangents and solutions")
    ap.add_argument("--layouts", type=int, default=200)
    ap.add_argument("--epochs", type=int, default=3)
    ap.add_argument("--batch", type=int, default=64)
    ap.add_argument("--lr", type=float, default=2e-3)
    args = ap.parse_args()
    ctx = api.Context(0)
    gnn, losses = train_default(ctx, n_layouts=args.layouts, n_batch=args.batch, epochs=args.epochs, lr=args.lr,
                                dump=args.dump)
    gnn.save(args.out, losses=losses.astype(np.float32), layouts=args.layouts, epochs=args.epochs,
             batch=args.batch, size=np.array([128, 32, 32]))
    print(f"saved {args.out}: final loss {losses[-20:].mean():.4e} (first {losses[:8].mean():.4e})")


if __name__ == "__main__":
    main()

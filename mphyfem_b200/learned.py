"""Learned factorised preconditioner (MPHY_PC_FSAI_LEARNED): parameter initialisation, GPU
training on operators the solver assembles, and persistence of the trained weights.

The network (csrc/gnn.cu) predicts the blocks of G in M = G^T G from the Jacobi-scaled operator,
as a correction to block-Jacobi FSAI (so an untrained network is block-Jacobi). Training minimises
Kaporin's condition number of G A G^T (the functional exact FSAI minimises), so it needs no
targets. Training runs
entirely in libmphy.so's forward/backward/Adam kernels; this module only orders the steps.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from . import _lib as L

H, LAYERS, NIN = 64, 3, 13
DEFAULT_WEIGHTS = os.path.join(os.path.dirname(os.path.abspath(__file__)), "data", "fsai_gnn.npz")


def param_count() -> int:
    return int(L.load().mphy_gnn_param_count())


def init_params(seed: int = 0) -> np.ndarray:
    """Uniform fan-in initialisation (bound 1/sqrt(fan_in)), biases zero; decoder small."""
    rng = np.random.Generator(np.random.PCG64(seed))
    parts = []

    def lin(o, k, scale=1.0):
        parts.append(rng.uniform(-1, 1, size=o * k) * scale / np.sqrt(k))

    def zeros(n):
        parts.append(np.zeros(n))
    lin(H, NIN)
    zeros(H)
    for _ in range(LAYERS):
        lin(H, H)          # U
        lin(H, 9)          # V
        zeros(H)           # c
        lin(H, H, 0.5)     # S
        lin(H, H, 0.5)     # T
        zeros(H)           # d
    lin(9, H, 0.1)         # Wa
    lin(9, H, 0.1)         # Wb
    zeros(81)              # Wc
    # zero decoder weights: the network starts as block-Jacobi FSAI (a valid SPD preconditioner)
    zeros(9)
    p = np.concatenate(parts).astype(np.float32)
    assert p.size == param_count(), (p.size, param_count())
    return p


class Gnn:
    """The network on one device (wraps mphy_gnn_*)."""

    def __init__(self, ctx, params: np.ndarray | None = None, seed: int = 0):
        self.ctx, self.lib = ctx, ctx.lib
        p = np.ascontiguousarray(init_params(seed) if params is None else params, np.float32)
        h = C.c_void_p()
        L.check(self.lib.mphy_gnn_create(ctx.h, p.ctypes.data_as(C.POINTER(C.c_float)), C.byref(h)))
        self.h = h

    @property
    def params(self) -> np.ndarray:
        p = np.zeros(param_count(), np.float32)
        L.check(self.lib.mphy_gnn_get_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))
        return p

    @params.setter
    def params(self, p):
        p = np.ascontiguousarray(p, np.float32)
        L.check(self.lib.mphy_gnn_set_params(self.h, p.ctypes.data_as(C.POINTER(C.c_float))))

    def loss_and_grads(self, solver):
        g = np.zeros(param_count(), np.float32)
        loss = C.c_double()
        L.check(self.lib.mphy_gnn_loss_and_grads(self.h, solver.h, C.byref(loss), g.ctypes.data_as(C.POINTER(C.c_float))))
        return loss.value, g

    def train_step(self, solver, lr: float) -> float:
        loss = C.c_double()
        L.check(self.lib.mphy_gnn_train_step(self.h, solver.h, float(lr), C.byref(loss)))
        return loss.value

    def predict(self, solver) -> float:
        ms = C.c_float()
        L.check(self.lib.mphy_gnn_predict(self.h, solver.h, C.byref(ms)))
        return ms.value

    def attach(self, solver):
        L.check(self.lib.mphy_solver_attach_gnn(solver.h, self.h))

    def save(self, path: str = DEFAULT_WEIGHTS, **meta):
        os.makedirs(os.path.dirname(path), exist_ok=True)
        np.savez_compressed(path, params=self.params, **{k: np.asarray(v) for k, v in meta.items()})

    def close(self):
        if getattr(self, "h", None):
            self.lib.mphy_gnn_destroy(self.h)
            self.h = None

    def __del__(self):
        self.close()


def load_params(path: str = DEFAULT_WEIGHTS) -> np.ndarray:
    return np.load(path)["params"].astype(np.float32)


def training_problems(n_layouts: int, size=(32, 8, 8), seed0: int = 100, with_batched: int = 0):
    """Seeded two-phase inclusion layouts (radii scaled to the mesh) plus batched blocks."""
    from . import meshgen
    nx, ny, nz = size
    h = 1.0 / ny
    out = [meshgen.two_phase_inclusions(nx, ny, nz, seed=seed0 + i, r_range=(1.5 * h, min(3.0 * h, 0.45)))
           for i in range(n_layouts)]
    if with_batched:
        out += meshgen.batched_blocks(with_batched, seed=11)
    return out


def train(ctx, problems, steps: int, lr: float = 1e-3, gnn: Gnn | None = None, precision: int | None = None,
          log=None):
    """Round-robin Adam steps over the problems (operators assembled at u = 0). Returns (gnn, losses)."""
    import torch
    from . import api
    gnn = gnn or Gnn(ctx)
    prec = L.PREC_MIXED if precision is None else precision
    solvers = []
    for p in problems:
        mesh = api.Mesh(ctx, p)
        sol = api.SolverGpu(mesh, api.Pattern(mesh), pc_type=L.PC_FSAI_LEARNED, precision=prec)
        sol.calcStiffnessAndResidual(torch.zeros(p.n_dof, dtype=torch.float64, device="cuda"))
        solvers.append(sol)
    losses = []
    for it in range(steps):
        losses.append(gnn.train_step(solvers[it % len(solvers)], lr))
        if log and (it % 50 == 0 or it == steps - 1):
            log(f"step {it} loss {losses[-1]:.4e}")
    return gnn, np.array(losses)

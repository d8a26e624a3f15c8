"""Learned FSAI: GPU forward/backward against the FP64 torch restatement, training, and what the
trained network gains over Jacobi-PCG (the method without it), with the true-residual fallback.

Loss: Kaporin's condition number of the preconditioned operator. Tolerances: loss within 1e-4
relative; every parameter tensor's gradient within 2e-3 relative (FP32 atomics and FP32 features
on the GPU against FP64 on the CPU, same BF16 weights)."""
import numpy as np
import pytest

from mphyfem_b200 import meshgen

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def env():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from mphyfem_b200 import _lib, api, build, learned
    build.build()
    return torch, api, _lib, learned, api.Context(0)


def _assembled(torch, api, _lib, ctx, p, prec):
    mesh = api.Mesh(ctx, p)
    pat = api.Pattern(mesh)
    sol = api.SolverGpu(mesh, pat, pc_type=_lib.PC_FSAI_LEARNED, precision=prec)
    sol.calcStiffnessAndResidual(torch.zeros(p.n_dof, dtype=torch.float64, device="cuda"))
    return mesh, pat, sol


@pytest.mark.parametrize("prec", ["PREC_FP64", "PREC_MIXED"])
def test_gnn_loss_and_gradients_match_oracle(env, prec):
    from oracle import fsai_ref, gnn_ref
    torch, api, _lib, learned, ctx = env
    p = meshgen.two_phase_inclusions(8, 3, 3, seed=5, r_range=(0.3, 0.45))
    mesh, pat, sol = _assembled(torch, api, _lib, ctx, p, getattr(_lib, prec))
    params = learned.init_params(seed=1)
    gnn = learned.Gnn(ctx, params)
    loss, grads = gnn.loss_and_grads(sol)
    lrow, lcol = sol.pc_pattern()
    val, _, _ = sol.export(want_rhs=False, want_reac=False)
    rp, col = pat.export_csr()
    A = fsai_ref.full_operator(p.n_node, p.fixed, rp, col, val)
    nbrs = fsai_ref.node_neighbours(p.conn, p.n_node)
    loss_ref, grads_ref, _ = gnn_ref.loss_and_grads(params, A, p.fixed, nbrs, lrow, lcol)
    assert abs(loss - loss_ref) <= 1e-4 * max(abs(loss_ref), 1.0)
    off, _ = gnn_ref.layout()
    for name, (o, n) in off.items():
        g, r = grads[o:o + n], grads_ref[o:o + n]
        assert np.linalg.norm(g - r) <= 2e-3 * max(np.linalg.norm(r), 1e-12), name


@pytest.fixture(scope="module")
def trained(env):
    torch, api, _lib, learned, ctx = env
    train = learned.training_problems(4, size=(24, 6, 6), seed0=200)
    return learned.train(ctx, train, steps=400, lr=2e-3)


def test_training_reduces_loss(trained):
    _, losses = trained
    # log K falls from its block-Jacobi start (zero decoder weights)
    assert losses[-20:].mean() < losses[:4].mean() - 0.02, (losses[:4], losses[-20:])


# FP64: rtol 1e-10. Mixed: the FP32-stored operator bounds the FP64 true residual near 1e-9 without
# refinement sweeps, so the tolerance is 1e-8 there.
@pytest.mark.parametrize("precision,rtol", [(0, 1e-10), (1, 1e-8)], ids=["fp64", "mixed"])
def test_learned_beats_jacobi(env, trained, precision, rtol):
    torch, api, _lib, learned, ctx = env
    gnn, _ = trained
    # held-out layout: learned FSAI-PCG against Jacobi-PCG, same true-residual tolerance
    q = meshgen.two_phase_inclusions(24, 6, 6, seed=999, r_range=(1.5 / 6, 3.0 / 6 * 0.9))
    its, xs = {}, {}
    for name, pc in (("jacobi", _lib.PC_JACOBI), ("learned", _lib.PC_FSAI_LEARNED)):
        mesh = api.Mesh(ctx, q)
        sol = api.SolverGpu(mesh, api.Pattern(mesh), pc_type=pc, precision=precision, rtol=rtol, norm_type=1)
        if pc == _lib.PC_FSAI_LEARNED:
            gnn.attach(sol)
        sol.calcStiffnessAndResidual(torch.zeros(q.n_dof, dtype=torch.float64, device="cuda"))
        sol.addExternalForces(torch.tensor(q.fnodal, device="cuda"), 0.2)
        rc, its[name], _ = sol.factoriseAndSolve()
        assert rc == 0
        if name == "learned":
            info = sol.pc_last()
            assert not info["fallback"], info
        assert sol.true_residual() <= 100 * rtol   # the acceptance bound of learned solves
        xs[name] = sol.solution().cpu().numpy()
    assert its["learned"] < 0.8 * its["jacobi"], its
    if precision == 0:
        assert np.linalg.norm(xs["learned"] - xs["jacobi"]) <= 1e-7 * np.linalg.norm(xs["jacobi"])


@pytest.mark.parametrize("coarse", [0, 16], ids=["local", "with_coarse"])
def test_learned_against_the_fsai_baselines(env, trained, coarse):
    """What the trained network gains, on the held-out layout, against the preconditioners it sits
    between: block-Jacobi FSAI (the network with zero weights, its starting point) and exact FSAI
    (the minimiser of the Kaporin functional it is trained on), alone and with the rigid-body
    coarse space. Every solve reaches the same FP64 true residual."""
    torch, api, _lib, learned, ctx = env
    gnn, _ = trained
    zero = learned.Gnn(ctx, np.zeros(learned.param_count(), np.float32))
    q = meshgen.two_phase_inclusions(24, 6, 6, seed=999, r_range=(1.5 / 6, 3.0 / 6 * 0.9))
    its = {}
    for name, pc, net in (("jacobi", _lib.PC_JACOBI, None), ("block_jacobi_fsai", _lib.PC_FSAI_LEARNED, zero),
                          ("learned", _lib.PC_FSAI_LEARNED, gnn), ("exact_fsai", _lib.PC_FSAI, None)):
        mesh = api.Mesh(ctx, q)
        sol = api.SolverGpu(mesh, api.Pattern(mesh), pc_type=pc, precision=0, rtol=1e-10, norm_type=1,
                            coarse_aggregates=coarse)
        if net is not None:
            net.attach(sol)
        sol.calcStiffnessAndResidual(torch.zeros(q.n_dof, dtype=torch.float64, device="cuda"))
        sol.addExternalForces(torch.tensor(q.fnodal, device="cuda"), 0.2)
        rc, its[name], _ = sol.factoriseAndSolve()
        assert rc == 0
        if net is not None:
            assert not sol.pc_last()["fallback"], name
        assert sol.true_residual() <= 100 * 1e-10
    assert its["learned"] < its["block_jacobi_fsai"], its
    assert its["exact_fsai"] < its["block_jacobi_fsai"], its
    assert its["block_jacobi_fsai"] <= its["jacobi"], its


def test_untrained_network_is_block_jacobi(env):
    """Zero weights: the prediction is block-Jacobi FSAI, the exact block FSAI on the diagonal
    pattern (G_nn = L^T, L L^T = A_nn^-1), so G A G^T has identity diagonal blocks."""
    torch, api, _lib, learned, ctx = env
    q = meshgen.hex8_cantilever(8, 2, 2)
    mesh, pat, sol = _assembled(torch, api, _lib, ctx, q, _lib.PREC_FP64)
    gnn = learned.Gnn(ctx, np.zeros(learned.param_count(), np.float32))
    gnn.predict(sol)
    G = sol.pc_get_blocks().cpu().numpy().reshape(-1, 3, 3)
    lrow, lcol = sol.pc_pattern()
    rows = np.repeat(np.arange(q.n_node), np.diff(lrow))
    val, _, _ = sol.export(want_rhs=False, want_reac=False)
    rp, col = pat.export_csr()
    from oracle import fsai_ref
    A = fsai_ref.full_operator(q.n_node, q.fixed, rp, col, val).tocsr()
    for j, (n, m) in enumerate(zip(rows, lcol)):
        if n != m:
            assert np.abs(G[j]).max() < 1e-6
            continue
        Ann = A[3 * n:3 * n + 3, 3 * n:3 * n + 3].toarray()
        # G is stored in BF16 (2^-9 relative rounding)
        np.testing.assert_allclose(G[j] @ Ann @ G[j].T, np.eye(3), atol=2e-2)


def test_useless_network_falls_back_to_jacobi(env):
    torch, api, _lib, learned, ctx = env
    q = meshgen.hex8_cantilever(12, 3, 3)
    from oracle import gnn_ref
    off, _ = gnn_ref.layout()
    p = np.zeros(learned.param_count(), np.float32)
    o, n = off["bo"]
    p[o:o + n] = np.nan  # a corrupted weights file: every predicted block is NaN
    gnn = learned.Gnn(ctx, p)
    mesh = api.Mesh(ctx, q)
    sol = api.SolverGpu(mesh, api.Pattern(mesh), pc_type=_lib.PC_FSAI_LEARNED, rtol=1e-10)
    gnn.attach(sol)
    sol.calcStiffnessAndResidual(torch.zeros(q.n_dof, dtype=torch.float64, device="cuda"))
    sol.addExternalForces(torch.tensor(q.fnodal, device="cuda"), 0.2)
    rc, its, _ = sol.factoriseAndSolve()
    assert rc == 0 and sol.pc_last()["fallback"]
    assert sol.true_residual() < 1e-8

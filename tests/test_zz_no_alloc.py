"""The allocation-free element evaluation (mphy_elem_eval_noalloc) against mphy_elem_eval.

Callers that cannot let the library call cudaMalloc -- their mesh already sits in device memory
under their own allocator, or they run under a no-allocation policy -- pass their device arrays
straight in; the scratch lives in a fixed array inside libmphy.so. This file is collected last
so that a run stopping at the first failure has already run every other test.
"""
import ctypes as C

import numpy as np
import pytest

from mphyfem_b200 import meshgen

pytestmark = pytest.mark.gpu

TOL = 1e-12  # relative to the largest entry, as in the other element parity tests


@pytest.fixture(scope="module")
def setup():
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from mphyfem_b200 import _lib, api, build
    build.build()
    return torch, api, _lib


def _call_noalloc(torch, api, _lib, ctx, p, mats, disp, tangent=0):
    def dev(a, dt):
        # at least one entry, so that an empty element list still passes valid (non-null) pointers
        a = np.ascontiguousarray(a).ravel()
        t = torch.zeros(max(a.size, 1), dtype=dt, device="cuda")
        t[:a.size] = torch.as_tensor(a, dtype=dt)
        return t
    coords = dev(p.coords, torch.float64)
    conn = dev(p.conn, torch.int32)
    mat_id = dev(p.mat_id, torch.int32)
    m = dev(mats, torch.float64)
    u = dev(disp, torch.float64)
    ns = 3 * p.npe
    Ke = torch.full((max(p.n_elem, 1), ns, ns), float("nan"), dtype=torch.float64, device="cuda")
    Re = torch.full((max(p.n_elem, 1), ns), float("nan"), dtype=torch.float64, device="cuda")
    bad = C.c_int64(123)
    ptr = lambda t: C.c_void_p(t.data_ptr())  # noqa: E731
    rc = ctx.lib.mphy_elem_eval_noalloc(ctx.h, p.n_node, ptr(coords), p.n_elem, p.npe, ptr(conn), ptr(mat_id),
                                        len(mats), ptr(m), ptr(u), tangent, ptr(Ke), ptr(Re), C.byref(bad))
    return rc, Ke[:p.n_elem].cpu().numpy(), Re[:p.n_elem].cpu().numpy(), bad.value


def _reference(torch, api, p, disp, tangent=0):
    ctx = api.Context(0)
    mesh = api.Mesh(ctx, p)
    Ke, Re, bad = api.calc_stiffness_and_residual(mesh, torch.tensor(disp, device="cuda"), tangent)
    return Ke.cpu().numpy(), Re.cpu().numpy(), bad


def _close(a, b):
    return np.abs(a - b).max() <= TOL * max(np.abs(b).max(), 1e-300)


def test_noalloc_matches_elem_eval_two_calls_in_a_row(setup):
    torch, api, _lib = setup
    ctx = api.Context(0)
    rng = np.random.default_rng(7)
    # call 1: hex8 two-material block; call 2: tet10 with other materials and tangent
    p1 = meshgen.two_phase_inclusions(12, 4, 4, seed=3, r_range=(0.15, 0.3), vol_frac=0.2)
    u1 = 0.01 * rng.standard_normal(p1.n_dof) * (p1.fixed == 0)
    p2 = meshgen.tet10_kuhn(3, 2, 2, lx=1.5)
    p2.mats = np.stack([meshgen.nh_material(0.4, 30.0), meshgen.nh_material(2.0, 5.0, utype=4)])
    p2.mat_id = (np.arange(p2.n_elem) % 2).astype(np.int32)
    u2 = 0.01 * rng.standard_normal(p2.n_dof) * (p2.fixed == 0)
    for p, u, tangent in ((p1, u1, 0), (p2, u2, 1)):
        rc, Ke, Re, bad = _call_noalloc(torch, api, _lib, ctx, p, p.mats, u, tangent)
        assert rc == _lib.OK and bad == -1
        Kr, Rr, br = _reference(torch, api, p, u, tangent)
        assert br == -1
        assert _close(Ke, Kr) and _close(Re, Rr)


def test_noalloc_flags_reset_between_calls_and_limits(setup):
    torch, api, _lib = setup
    ctx = api.Context(0)
    p = meshgen.hex8_cantilever(4, 2, 2)
    u = np.zeros((p.n_node, 3))
    for a in (1, 2, 5, 6):  # fold element 3 through itself
        u[p.conn[3, a], 0] = -3.0 * (p.coords[p.conn[3, a], 0] - p.coords[p.conn[3, 0], 0])
    rc, _, _, bad = _call_noalloc(torch, api, _lib, ctx, p, p.mats, u.ravel())
    assert rc == _lib.ERR_NEG_JACOBIAN and 0 <= bad <= 3
    _, _, bref = _reference(torch, api, p, u.ravel())
    assert bad == bref
    # the next call on a valid state must not see the previous call's flag
    rc, Ke, Re, bad = _call_noalloc(torch, api, _lib, ctx, p, p.mats, np.zeros(p.n_dof))
    assert rc == _lib.OK and bad == -1
    Kr, Rr, _ = _reference(torch, api, p, np.zeros(p.n_dof))
    assert _close(Ke, Kr)
    # more materials than the fixed scratch holds, and out-of-range material ids, are refused
    many = np.tile(p.mats, (1025, 1))
    rc, _, _, _ = _call_noalloc(torch, api, _lib, ctx, p, many, np.zeros(p.n_dof))
    assert rc == _lib.ERR_INVALID_ARG
    q = meshgen.hex8_cantilever(4, 2, 2)
    q.mat_id = q.mat_id.copy()
    q.mat_id[5] = 1
    rc, _, _, _ = _call_noalloc(torch, api, _lib, ctx, q, q.mats, np.zeros(q.n_dof))
    assert rc == _lib.ERR_INVALID_ARG


def test_noalloc_largest_table_empty_mesh_and_bad_material(setup):
    torch, api, _lib = setup
    ctx = api.Context(0)
    p = meshgen.hex8_cantilever(4, 2, 2)
    rng = np.random.default_rng(11)
    u = 0.01 * rng.standard_normal(p.n_dof) * (p.fixed == 0)
    # the largest table the fixed scratch holds: 1024 rows, every element on the last one
    mats = np.tile(meshgen.nh_material(1.0, 10.0), (1024, 1))
    mats[1023] = meshgen.nh_material(0.7, 25.0, utype=4)
    q = meshgen.hex8_cantilever(4, 2, 2)
    q.mats = mats[1023:1024].copy()
    q.mat_id = np.zeros(q.n_elem, dtype=np.int32)
    p.mat_id = np.full(p.n_elem, 1023, dtype=np.int32)
    rc, Ke, Re, bad = _call_noalloc(torch, api, _lib, ctx, p, mats, u)
    assert rc == _lib.OK and bad == -1
    Kr, Rr, br = _reference(torch, api, q, u)
    assert br == -1 and _close(Ke, Kr) and _close(Re, Rr)
    # an empty element list launches no element kernel and reports no bad element
    e = meshgen.hex8_cantilever(4, 2, 2)
    e.conn = e.conn[:0]
    e.mat_id = e.mat_id[:0]
    rc, Ke, Re, bad = _call_noalloc(torch, api, _lib, ctx, e, e.mats, np.zeros(e.n_dof))
    assert rc == _lib.OK and bad == -1 and Ke.size == 0
    # a material row with Kinv = 0 is refused, as mphy_mesh_create refuses it
    z = meshgen.hex8_cantilever(4, 2, 2)
    zm = np.stack([meshgen.nh_material(1.0, 10.0), meshgen.nh_material(1.0, 10.0)])
    zm[1, 1] = 0.0
    rc, _, _, _ = _call_noalloc(torch, api, _lib, ctx, z, zm, np.zeros(z.n_dof))
    assert rc == _lib.ERR_INVALID_ARG

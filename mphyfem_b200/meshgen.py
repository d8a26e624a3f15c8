"""Seeded synthetic meshes and load cases for the femSolidmechanics Newton-step workloads.

The reference reads Gmsh 2.2 meshes plus a block-structured ``config`` file
(src/utilities/femBase.cpp:121-476). The workloads here are generated in memory with the
same conventions so that the product path, the oracle and (where it can be built) the
reference all see identical inputs:

* hex8 node order (-,-,-),(+,-,-),(+,+,-),(-,+,-),(-,-,+),(+,-,+),(+,+,+),(-,+,+)
  (src/utilities/BasisFunctionsLagrange.cpp:1243-1250);
* tet10 node order: 4 vertices, then mid-side nodes of edges (0,1),(1,2),(0,2),(0,3),(2,3),(1,3)
  (BasisFunctionsLagrange.cpp:912-921, equal to the Gmsh order);
* the cantilever's long axis is x; the face x = 0 is clamped ("fixed" patch,
  src/femSolidmechanics/femSolidmechanics1.cpp:1479-1543) and a uniform traction on the face
  x = L is applied as consistent nodal forces (``Nodal Forces`` block,
  src/utilities/femBase.cpp:876-919; each quad face corner receives t * A_face / 4, each
  tri6 face node its consistent share);
* Neo-Hookean material rows are ``(mu, Kinv, Utype)`` with Utype 3, U = K/2 (J-1)^2
  (src/material/MaterialBase.cpp:107-116).

Node numbering is x-fastest so that consecutive elements share nodes, which keeps the
assembly's scatter traffic L2-resident on the GPU.
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

HEX8_CORNERS = np.array(
    [[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]],
    dtype=np.int64,
)
# Kuhn split of a hex (hex8 corner indices) into 6 tets around the 0-6 diagonal.
KUHN_TETS = np.array(
    [[0, 1, 2, 6], [0, 2, 3, 6], [0, 3, 7, 6], [0, 7, 4, 6], [0, 4, 5, 6], [0, 5, 1, 6]],
    dtype=np.int64,
)
TET10_EDGES = np.array([[0, 1], [1, 2], [0, 2], [0, 3], [2, 3], [1, 3]], dtype=np.int64)


@dataclass
class Problem:
    """One solid-mechanics problem: mesh, materials, constraints and reference loads."""

    name: str
    coords: np.ndarray  # [n_node, 3] float64
    conn: np.ndarray  # [n_elem, npe] int32
    mat_id: np.ndarray  # [n_elem] int32 (0-based material index)
    mats: np.ndarray  # [n_mat, 3] float64 rows (mu, Kinv, Utype)
    fixed: np.ndarray  # [n_node*3] uint8, 1 = prescribed (zero) displacement
    fnodal: np.ndarray  # [n_node*3] float64 nodal forces at load factor 1
    dt: float = 0.2
    t_final: float = 1.0
    max_steps: int = 5
    newton_rtol: float = 1e-10
    cg_rtol: float = 1e-12
    meta: dict = field(default_factory=dict)
    mat_model: np.ndarray | None = None  # [n_mat] int32 hyperelastic model per material (None: Neo-Hookean)
    mat_data: np.ndarray | None = None  # [n_mat, 4] float64 model parameters (mu; c1 c2; mu Im; mu N)
    # prescribed displacement of every prescribed DOF at time t: t * presc_ramp + presc_const
    presc_ramp: np.ndarray | None = None  # [n_node*3] float64
    presc_const: np.ndarray | None = None  # [n_node*3] float64

    @property
    def n_node(self) -> int:
        return int(self.coords.shape[0])

    @property
    def n_elem(self) -> int:
        return int(self.conn.shape[0])

    @property
    def npe(self) -> int:
        return int(self.conn.shape[1])

    @property
    def n_dof(self) -> int:
        return 3 * self.n_node

    @property
    def n_free(self) -> int:
        return int(self.n_dof - int(self.fixed.sum()))


def nh_material(mu: float, kappa: float, utype: int = 3) -> np.ndarray:
    """Material row (mu, Kinv, Utype) for ``data_deviatoric mu`` / ``data_volumetric Utype 1/kappa``."""
    return np.array([mu, 1.0 / kappa, float(utype)], dtype=np.float64)


def _grid_nodes(nx: int, ny: int, nz: int, lx: float, ly: float, lz: float) -> np.ndarray:
    i = np.arange(nx + 1, dtype=np.float64) * (lx / nx)
    j = np.arange(ny + 1, dtype=np.float64) * (ly / ny)
    k = np.arange(nz + 1, dtype=np.float64) * (lz / nz)
    Z, Y, X = np.meshgrid(k, j, i, indexing="ij")
    return np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)


def _grid_cells(nx: int, ny: int, nz: int) -> np.ndarray:
    """[n_cell, 8] corner node ids of every cell in hex8 order, cells x-fastest."""
    ci, cj, ck = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ci, cj, ck = (a.transpose(2, 1, 0).ravel() for a in (ci, cj, ck))  # x fastest
    sx, sy = 1, nx + 1
    sz = (nx + 1) * (ny + 1)
    base = ci * sx + cj * sy + ck * sz
    off = HEX8_CORNERS[:, 0] * sx + HEX8_CORNERS[:, 1] * sy + HEX8_CORNERS[:, 2] * sz
    return (base[:, None] + off[None, :]).astype(np.int64)


def hex8_cantilever(nx: int, ny: int, nz: int, lx: float = 4.0, ly: float = 1.0, lz: float = 1.0,
                    traction=(0.0, 0.0, -0.05), mu: float = 1.0, kappa: float = 10.0,
                    name: str | None = None) -> Problem:
    """Structured hex8 block [0,lx]x[0,ly]x[0,lz], clamped at x=0, traction on x=lx."""
    coords = _grid_nodes(nx, ny, nz, lx, ly, lz)
    conn = _grid_cells(nx, ny, nz).astype(np.int32)
    n_node = coords.shape[0]
    fixed = np.zeros((n_node, 3), dtype=np.uint8)
    fixed[np.isclose(coords[:, 0], 0.0)] = 1
    fnodal = np.zeros((n_node, 3), dtype=np.float64)
    # consistent nodal forces of a uniform traction on the x = lx face (quad4 faces)
    area = (ly / ny) * (lz / nz)
    t = np.asarray(traction, dtype=np.float64)
    j, k = np.meshgrid(np.arange(ny), np.arange(nz), indexing="ij")
    for dj, dk in ((0, 0), (1, 0), (1, 1), (0, 1)):
        nid = nx + (nx + 1) * ((j + dj) + (ny + 1) * (k + dk))
        np.add.at(fnodal, nid.ravel(), t * (area / 4.0))
    return Problem(
        name=name or f"hex8_{nx}x{ny}x{nz}",
        coords=coords, conn=conn, mat_id=np.zeros(conn.shape[0], np.int32),
        mats=nh_material(mu, kappa)[None, :], fixed=fixed.ravel(), fnodal=fnodal.ravel(),
        meta={"nx": nx, "ny": ny, "nz": nz, "traction": list(map(float, t))},
    )


def cantilever_small() -> Problem:
    """Plain method, small: 32(x) x 8 x 8 hex8 on [0,4]x[0,1]^2, 2048 elements, 8019 DOFs."""
    return hex8_cantilever(32, 8, 8, name="hex8_cantilever_32x8x8")


def cantilever_large() -> Problem:
    """Precision form at scale: 256(x) x 64 x 64 hex8, 1,048,576 elements, 3,257,475 DOFs."""
    p = hex8_cantilever(256, 64, 64, name="hex8_cantilever_256x64x64")
    p.newton_rtol = 1e-8
    return p


def tet10_kuhn(nx: int, ny: int, nz: int, lx: float = 4.0, ly: float = 1.0, lz: float = 1.0,
               jitter: float = 0.1, seed: int = 7, traction=(0.0, 0.0, -0.02), mu: float = 1.0,
               kappa: float = 100.0, name: str | None = None) -> Problem:
    """Kuhn-split tet10 block: each hex cell is cut into 6 tets around its 0-6 diagonal,
    interior vertices jittered by U(-jitter*h, jitter*h) per coordinate (numpy PCG64(seed),
    drawn in node-index order), mid-side nodes at exact edge midpoints."""
    verts = _grid_nodes(nx, ny, nz, lx, ly, lz)
    h = np.array([lx / nx, ly / ny, lz / nz])
    rng = np.random.Generator(np.random.PCG64(seed))
    jit = rng.uniform(-jitter, jitter, size=verts.shape) * h[None, :]
    interior = (
        (verts[:, 0] > 1e-12) & (verts[:, 0] < lx - 1e-12)
        & (verts[:, 1] > 1e-12) & (verts[:, 1] < ly - 1e-12)
        & (verts[:, 2] > 1e-12) & (verts[:, 2] < lz - 1e-12)
    )
    verts = verts + jit * interior[:, None]
    cells = _grid_cells(nx, ny, nz)
    tets = cells[:, KUHN_TETS].reshape(-1, 4)
    # positive orientation in the reference tet's (xi1, xi2, xi3) = (v1-v0, v2-v0, v3-v0) frame
    a = verts[tets[:, 1]] - verts[tets[:, 0]]
    b = verts[tets[:, 2]] - verts[tets[:, 0]]
    c = verts[tets[:, 3]] - verts[tets[:, 0]]
    neg = np.einsum("ij,ij->i", np.cross(a, b), c) < 0
    tets[neg, 1], tets[neg, 2] = tets[neg, 2].copy(), tets[neg, 1].copy()
    # unique edges -> mid-side node ids numbered after the vertices, in sorted edge order
    e = tets[:, TET10_EDGES]  # [n_tet, 6, 2]
    lo, hi = np.minimum(e[..., 0], e[..., 1]), np.maximum(e[..., 0], e[..., 1])
    key = lo.astype(np.int64) * verts.shape[0] + hi
    ukey, inv = np.unique(key.ravel(), return_inverse=True)
    mid_id = verts.shape[0] + inv.reshape(key.shape)
    ulo, uhi = ukey // verts.shape[0], ukey % verts.shape[0]
    coords = np.concatenate([verts, 0.5 * (verts[ulo] + verts[uhi])], axis=0)
    conn = np.concatenate([tets, mid_id], axis=1).astype(np.int32)
    n_node = coords.shape[0]
    fixed = np.zeros((n_node, 3), dtype=np.uint8)
    fixed[np.abs(coords[:, 0]) < 1e-12] = 1
    # consistent nodal forces of a uniform traction on tri6 faces of the x = lx face:
    # a flat tri6 with area A gives 0 to each vertex and A/3 to each mid-side node
    t = np.asarray(traction, dtype=np.float64)
    fnodal = np.zeros((n_node, 3), dtype=np.float64)
    on_face = np.abs(coords[:, 0] - lx) < 1e-12
    faces_local = [(1, 2, 3, 5, 8, 9), (0, 2, 3, 6, 8, 7), (0, 1, 3, 4, 9, 7), (0, 1, 2, 4, 5, 6)]
    for fl in faces_local:
        fn = conn[:, fl]
        sel = on_face[fn].all(axis=1)
        fn = fn[sel]
        p0, p1, p2 = coords[fn[:, 0]], coords[fn[:, 1]], coords[fn[:, 2]]
        area = 0.5 * np.linalg.norm(np.cross(p1 - p0, p2 - p0), axis=1)
        for m in (3, 4, 5):
            np.add.at(fnodal, fn[:, m], (area / 3.0)[:, None] * t[None, :])
    return Problem(
        name=name or f"tet10_kuhn_{nx}x{ny}x{nz}",
        coords=coords, conn=conn, mat_id=np.zeros(conn.shape[0], np.int32),
        mats=nh_material(mu, kappa)[None, :], fixed=fixed.ravel(), fnodal=fnodal.ravel(),
        dt=0.1, max_steps=10, newton_rtol=1e-8, cg_rtol=1e-8,
        meta={"nx": nx, "ny": ny, "nz": nz, "seed": seed, "traction": list(map(float, t))},
    )


# 27-node hex node order (BasisFunctionsLagrange.cpp:1300-1399): the 1D indices (i, j, k) of each
# node, 0 at xi = -1, 1 at xi = +1, 2 at the midpoint (the 1D quadratic Lagrange order)
HEX27_IJK = np.array([
    [0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1],
    [2, 0, 0], [0, 2, 0], [0, 0, 2], [1, 2, 0], [1, 0, 2], [2, 1, 0], [1, 1, 2], [0, 1, 2],
    [2, 0, 1], [0, 2, 1], [1, 2, 1], [2, 1, 1], [2, 2, 0], [2, 0, 2], [0, 2, 2], [1, 2, 2],
    [2, 1, 2], [2, 2, 1], [2, 2, 2]], dtype=np.int64)


def hex27_cantilever(nx: int, ny: int, nz: int, lx: float = 4.0, ly: float = 1.0, lz: float = 1.0,
                     jitter: float = 0.0, seed: int = 7, traction=(0.0, 0.0, -0.02), mu: float = 1.0,
                     kappa: float = 100.0, name: str | None = None) -> Problem:
    """27-node hex block [0,lx]x[0,ly]x[0,lz] (the P2 displacement of Elem_Solid_3D_Mixed1's
    P2-P1 hex; its 8 corner nodes carry the pressure), clamped at x = 0, uniform traction on
    x = lx. Nodes sit on the (2nx+1)(2ny+1)(2nz+1) half-spacing grid, x fastest; interior grid
    nodes may be jittered by U(-jitter*h/2, jitter*h/2) per coordinate (numpy PCG64(seed)), which
    keeps every element's edges straight only when jitter = 0."""
    mx, my, mz = 2 * nx + 1, 2 * ny + 1, 2 * nz + 1
    gx, gy, gz = np.linspace(0.0, lx, mx), np.linspace(0.0, ly, my), np.linspace(0.0, lz, mz)
    Z, Y, X = np.meshgrid(gz, gy, gx, indexing="ij")
    coords = np.stack([X.ravel(), Y.ravel(), Z.ravel()], axis=1)
    if jitter > 0.0:
        h = np.array([lx / nx, ly / ny, lz / nz]) * 0.5
        rng = np.random.Generator(np.random.PCG64(seed))
        jit = rng.uniform(-jitter, jitter, size=coords.shape) * h[None, :]
        interior = ((coords[:, 0] > 1e-12) & (coords[:, 0] < lx - 1e-12) & (coords[:, 1] > 1e-12)
                    & (coords[:, 1] < ly - 1e-12) & (coords[:, 2] > 1e-12) & (coords[:, 2] < lz - 1e-12))
        coords = coords + jit * interior[:, None]
    off = np.array([0, 2, 1])  # grid offset of 1D index 0 (xi = -1), 1 (xi = +1), 2 (midpoint)
    ex, ey, ez = np.meshgrid(np.arange(nx), np.arange(ny), np.arange(nz), indexing="ij")
    ex, ey, ez = ex.transpose(2, 1, 0).ravel(), ey.transpose(2, 1, 0).ravel(), ez.transpose(2, 1, 0).ravel()
    gxi = 2 * ex[:, None] + off[HEX27_IJK[:, 0]][None, :]
    gyi = 2 * ey[:, None] + off[HEX27_IJK[:, 1]][None, :]
    gzi = 2 * ez[:, None] + off[HEX27_IJK[:, 2]][None, :]
    conn = (gxi + mx * (gyi + my * gzi)).astype(np.int32)
    n_node = coords.shape[0]
    fixed = np.zeros((n_node, 3), dtype=np.uint8)
    fixed[np.abs(coords[:, 0]) < 1e-12] = 1
    # consistent nodal forces of a uniform traction on the 9-node faces of x = lx: the 1D
    # quadratic weights (1/6, 2/3, 1/6) of each face edge, tensored
    t = np.asarray(traction, dtype=np.float64)
    fnodal = np.zeros((n_node, 3), dtype=np.float64)
    w1 = np.array([1.0 / 6.0, 2.0 / 3.0, 1.0 / 6.0])
    area = (ly / ny) * (lz / nz)
    for fy in range(ny):
        for fz in range(nz):
            for a in range(3):
                for b in range(3):
                    nid = (mx - 1) + mx * ((2 * fy + a) + my * (2 * fz + b))
                    fnodal[nid] += t * area * w1[a] * w1[b]
    return Problem(
        name=name or f"hex27_{nx}x{ny}x{nz}",
        coords=coords, conn=conn, mat_id=np.zeros(conn.shape[0], np.int32),
        mats=nh_material(mu, kappa)[None, :], fixed=fixed.ravel(), fnodal=fnodal.ravel(),
        dt=0.1, max_steps=10, newton_rtol=1e-8, cg_rtol=1e-8,
        meta={"nx": nx, "ny": ny, "nz": nz, "seed": seed, "traction": list(map(float, t)), "element": "hex27"},
    )


def tet10_near_incompressible() -> Problem:
    """Near-incompressible unstructured form: Kuhn tet10 on 96(x) x 48 x 48, kappa = 100."""
    return tet10_kuhn(96, 48, 48, name="tet10_kuhn_96x48x48")


def two_phase_inclusions(nx: int, ny: int, nz: int, seed: int = 23, vol_frac: float = 0.20,
                         r_range=(0.03, 0.08), mu_ratio: float = 1000.0, kappa_over_mu: float = 10.0,
                         traction=(0.0, 0.0, -0.05), name: str | None = None,
                         max_tries: int = 2_000_000) -> Problem:
    """hex8 cantilever with spherical stiff inclusions placed by random sequential addition
    (numpy PCG64(seed)) to the target volume fraction; an element is stiff when its centroid
    lies inside a sphere. Material 0 = matrix (mu 1), material 1 = inclusion (mu = mu_ratio)."""
    p = hex8_cantilever(nx, ny, nz, traction=traction, mu=1.0, kappa=kappa_over_mu,
                        name=name or f"hex8_two_phase_{nx}x{ny}x{nz}")
    lx, ly, lz = 4.0, 1.0, 1.0
    rng = np.random.Generator(np.random.PCG64(seed))
    cap = 1024
    cen, rad, n = np.empty((cap, 3)), np.empty(cap), 0
    vol, target, tries = 0.0, vol_frac * lx * ly * lz, 0
    while vol < target and tries < max_tries:
        tries += 1
        r = rng.uniform(*r_range)
        c = rng.uniform([r, r, r], [lx - r, ly - r, lz - r])
        if n:
            d = np.linalg.norm(cen[:n] - c, axis=1)
            if np.any(d < rad[:n] + r):
                continue
        if n == cap:
            cap *= 2
            cen = np.concatenate([cen, np.empty((cap - n, 3))])
            rad = np.concatenate([rad, np.empty(cap - n)])
        cen[n], rad[n] = c, r
        n += 1
        vol += 4.0 / 3.0 * np.pi * r ** 3
    centers, radii = list(cen[:n]), list(rad[:n])
    # element (i, j, k) of the structured grid has its centroid at ((i+.5)hx, (j+.5)hy, (k+.5)hz);
    # test only the cells inside each sphere's bounding box
    h = np.array([lx / nx, ly / ny, lz / nz])
    dims = np.array([nx, ny, nz])
    inside = np.zeros((nz, ny, nx), dtype=bool)
    for c, r in zip(centers, radii):
        lo = np.maximum(np.floor((c - r) / h - 0.5).astype(int), 0)
        hi = np.minimum(np.ceil((c + r) / h - 0.5).astype(int), dims - 1)
        ii = (np.arange(lo[0], hi[0] + 1) + 0.5) * h[0] - c[0]
        jj = (np.arange(lo[1], hi[1] + 1) + 0.5) * h[1] - c[1]
        kk = (np.arange(lo[2], hi[2] + 1) + 0.5) * h[2] - c[2]
        d2 = kk[:, None, None] ** 2 + jj[None, :, None] ** 2 + ii[None, None, :] ** 2
        inside[lo[2]:hi[2] + 1, lo[1]:hi[1] + 1, lo[0]:hi[0] + 1] |= d2 <= r * r
    inside = inside.ravel()  # cells are numbered x-fastest, like the elements
    p.mat_id = inside.astype(np.int32)
    p.mats = np.stack([nh_material(1.0, kappa_over_mu), nh_material(mu_ratio, kappa_over_mu * mu_ratio)])
    p.newton_rtol = 1e-8
    p.meta.update({"seed": seed, "n_spheres": len(radii), "vol_frac": float(vol / (lx * ly * lz)),
                   "stiff_elems": int(inside.sum())})
    return p


def batched_blocks(n_inst: int = 512, seed: int = 11):
    """Batched form: independent hex8 blocks, nx, ny ~ U{4..16}, nz ~ U{16..64}; per instance
    log mu ~ U(ln 0.1, ln 10), nu ~ U(0.30, 0.49), |t| ~ U(0.01, 0.08). The long axis (nz
    cells, length 4) is laid along x so the cantilever's clamp and load code applies unchanged;
    the problem is the same up to an axis relabelling. Returns a list of Problems."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for i in range(n_inst):
        nx, ny = (int(v) for v in rng.integers(4, 17, size=2))
        nz = int(rng.integers(16, 65))
        mu = float(np.exp(rng.uniform(np.log(0.1), np.log(10.0))))
        nu = float(rng.uniform(0.30, 0.49))
        tmag = float(rng.uniform(0.01, 0.08))
        kappa = 2.0 * mu * (1.0 + nu) / (3.0 * (1.0 - 2.0 * nu))
        q = hex8_cantilever(nz, nx, ny, lx=4.0, ly=1.0, lz=1.0, traction=(0.0, 0.0, -tmag),
                            mu=mu, kappa=kappa, name=f"block{i:03d}_{nx}x{ny}x{nz}")
        q.meta.update({"mu": mu, "nu": nu, "traction_mag": tmag, "kappa": kappa})
        out.append(q)
    return out


def batch_union(problems, name: str = "batch"):
    """Disjoint union of problems as one mesh: instance i owns nodes
    [inst_node_ptr[i], inst_node_ptr[i+1]), elements [inst_elem_ptr[i], inst_elem_ptr[i+1]) and
    material rows [inst_mat_ptr[i], inst_mat_ptr[i+1]). The load stepping (dt, t_final,
    max_steps) and tolerances are the first problem's; the instances must share npe."""
    problems = list(problems)
    assert problems and len({q.npe for q in problems}) == 1
    nptr = np.zeros(len(problems) + 1, np.int64)
    eptr = np.zeros(len(problems) + 1, np.int64)
    mptr = np.zeros(len(problems) + 1, np.int64)
    for i, q in enumerate(problems):
        nptr[i + 1] = nptr[i] + q.n_node
        eptr[i + 1] = eptr[i] + q.n_elem
        mptr[i + 1] = mptr[i] + len(q.mats)
    assert nptr[-1] < 2**31 // 3
    coords = np.concatenate([q.coords for q in problems])
    conn = np.concatenate([q.conn.astype(np.int64) + nptr[i] for i, q in enumerate(problems)]).astype(np.int32)
    mat_id = np.concatenate([q.mat_id.astype(np.int64) + mptr[i] for i, q in enumerate(problems)]).astype(np.int32)
    mats = np.concatenate([q.mats for q in problems])
    fixed = np.concatenate([q.fixed for q in problems]).astype(np.uint8)
    fnodal = np.concatenate([q.fnodal for q in problems])
    q0 = problems[0]
    model = data = None
    if any(q.mat_model is not None for q in problems):
        model = np.concatenate([q.mat_model if q.mat_model is not None else np.zeros(len(q.mats), np.int32)
                                for q in problems]).astype(np.int32)
        data = np.concatenate([_material_data(q) for q in problems])
    return Problem(name=name, coords=coords, conn=conn, mat_id=mat_id, mats=mats, fixed=fixed, fnodal=fnodal,
                   dt=q0.dt, t_final=q0.t_final, max_steps=q0.max_steps, newton_rtol=q0.newton_rtol,
                   cg_rtol=q0.cg_rtol,
                   meta={"inst_node_ptr": nptr.astype(np.int32), "inst_elem_ptr": eptr.astype(np.int32),
                         "inst_mat_ptr": mptr.astype(np.int32), "n_inst": len(problems)},
                   mat_model=model, mat_data=data)


def _material_data(q) -> np.ndarray:
    """[n_mat, 4] model parameters of a problem (Neo-Hookean rows: mu from mats)."""
    if q.mat_data is not None:
        return np.asarray(q.mat_data, np.float64).reshape(len(q.mats), 4)
    d = np.zeros((len(q.mats), 4))
    d[:, 0] = q.mats[:, 0]
    return d


def hyperelastic_material(model: int, data, kappa: float, utype: int = 3):
    """(mats row, model, data row) of one material: model 0 Neo-Hookean (mu), 1 Mooney-Rivlin
    (c1, c2), 2 Gent (mu, Im), 3 Arruda-Boyce (mu, N); data_volumetric Utype 1/kappa. The mats row
    carries data[0] in its first slot."""
    d = np.zeros(4)
    d[:len(data)] = data
    return np.array([d[0], 1.0 / kappa, float(utype)]), int(model), d

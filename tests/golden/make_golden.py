"""Generates tests/golden/cantilever_32x8x8.npz from the CPU oracle.

The reference cannot be built or run here (PETSc, Eigen, Boost, MPI, VTK are absent) and ships
no recorded outputs, so these fixtures are oracle outputs: they pin the oracle against
regressions and give the GPU parity tests fixed targets. Run from the repository root:

    python tests/golden/make_golden.py
"""
import hashlib
import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from mphyfem_b200 import meshgen  # noqa: E402
from oracle import binding  # noqa: E402


def probe_displacement(p, seed=5, amp=0.02):
    """Smooth bending-like field plus seeded noise, zero on the clamped face."""
    rng = np.random.Generator(np.random.PCG64(seed))
    x = p.coords
    u = np.zeros_like(x)
    s = x[:, 0] / x[:, 0].max()
    u[:, 2] = -0.3 * s * s
    u[:, 0] = 0.05 * s * (x[:, 2] - 0.5)
    u += amp * rng.standard_normal(u.shape) * s[:, None]
    return u.ravel()


def sha(a):
    return hashlib.sha256(np.ascontiguousarray(a).tobytes()).hexdigest()


def main():
    binding.build()
    p = meshgen.cantilever_small()
    op = binding.OracleProblem(p)
    afs, fav, rp, col = op.pattern()
    u = probe_displacement(p)
    val, rhs, reac, bad = op.assemble(u)
    assert bad == -1
    Ke, Re, _ = op.elements(u)
    sel = np.array([0, 1, 7, 100, 1023, 2047])
    binding.set_consistent_tangent(True)
    try:
        uc, hc = op.newton(max_newton=15)
    finally:
        binding.set_consistent_tangent(False)
    q = meshgen.cantilever_small()
    q.dt, q.max_steps = 0.1, 1
    oq = binding.OracleProblem(q)
    ur, hr = oq.newton(max_newton=10)
    out = dict(
        n_free=op.n_free, nnz=op.nnz, assy_sha=sha(afs.astype(np.int32)), fav_sha=sha(fav.astype(np.int32)),
        rowptr_sha=sha(rp.astype(np.int64)), col_sha=sha(col.astype(np.int32)),
        probe_u=u, probe_rhs=rhs, probe_reac=reac, probe_val_sum=float(val.sum()),
        probe_val_abs=float(np.abs(val).sum()), probe_diag=val[[int(np.searchsorted(col[rp[i]:rp[i + 1]], i)) + int(rp[i])
                                                                for i in range(op.n_free)]],
        probe_sel=sel, probe_Ke=Ke[sel], probe_Re=Re[sel],
        newton_consistent_hist=hc, newton_consistent_u=uc,
        newton_reference_step_hist=hr, newton_reference_step_u=ur,
    )
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "cantilever_32x8x8.npz")
    np.savez_compressed(path, **out)
    print("wrote", path, os.path.getsize(path), "bytes")


if __name__ == "__main__":
    main()

"""The product reading the reference's own input formats: a cantilever written as Gmsh 2.2 +
config with its load as a Tractions block solves to the same displacements as the generated
problem (whose load is the consistent nodal forces of the same traction)."""
import numpy as np
import pytest

from mphyfem_b200 import meshgen
from mphyfem_b200 import reference_io as rio

pytestmark = pytest.mark.gpu


def test_solve_from_reference_inputs(tmp_path):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    from mphyfem_b200 import api, build
    build.build()
    ctx = api.Context(0)
    p = meshgen.hex8_cantilever(16, 4, 4)
    clamp = rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 0.0))
    # load face ordered so dx/dxi1 runs along z: t = s1 dx/dxi1 = (0, 0, -0.05)
    load = [[f[0], f[3], f[2], f[1]] for f in rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 4.0))]
    hz = 1.0 / 4
    p.newton_rtol = 1e-9
    rio.write_gmsh22(tmp_path / "m.msh", p, {"clamp": clamp, "load": load})
    rio.write_config(tmp_path / "config", "m.msh", p, fixed_patches=("clamp",), nodal_forces=False,
                     tractions={"load": (0.0, -0.05 / (hz / 2.0), 0.0)})
    fem = api.FemSolidmechanicsGpu.from_reference_inputs(tmp_path / "config", ctx, tangent=1, rtol=1e-12)
    ref = api.FemSolidmechanicsGpu(p, ctx, tangent=1, rtol=1e-12)
    a = fem.solveWithNewtonRaphson(max_newton=15, tol_rel=1e-9)
    b = ref.solveWithNewtonRaphson(max_newton=15, tol_rel=1e-9)
    assert a.status == 0 and b.status == 0
    assert np.abs(a.disp - b.disp).max() <= 1e-10 * np.abs(b.disp).max()
    c = fem.solve_reference()          # the config's absolute tolerance (1e-9 here)
    assert c.status == 0 and c.hist[-1, 2] < 1e-9

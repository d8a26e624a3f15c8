"""The reference's input formats (Gmsh 2.2 + config): round trips of the generated workloads,
traction quadrature against closed forms, and the config reader's rules and limits."""
import os

import numpy as np
import pytest

from mphyfem_b200 import meshgen
from mphyfem_b200 import reference_io as rio


def _write(tmp_path, prob, patches, fixed=("clamp",), **kw):
    rio.write_gmsh22(tmp_path / "m.msh", prob, patches)
    rio.write_config(tmp_path / "config", "m.msh", prob, fixed_patches=fixed, **kw)
    return rio.read_config(tmp_path / "config")


@pytest.mark.parametrize("make", [lambda: meshgen.hex8_cantilever(8, 2, 3),
                                  lambda: meshgen.two_phase_inclusions(16, 4, 4, seed=3, r_range=(0.2, 0.3)),
                                  lambda: meshgen.tet10_kuhn(4, 2, 2)], ids=["hex8", "two_phase", "tet10"])
def test_round_trip(tmp_path, make):
    p = make()
    clamp = rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 0.0))
    q = _write(tmp_path, p, {"clamp": clamp})
    assert np.array_equal(q.coords, p.coords) and np.array_equal(q.conn, p.conn)
    assert np.array_equal(q.fixed, p.fixed)
    assert np.array_equal(q.fnodal, p.fnodal)
    # materials are renumbered by first use; the per-element rows must agree
    assert np.array_equal(q.mats[q.mat_id], p.mats[p.mat_id])
    assert (q.dt, q.t_final, q.max_steps) == (p.dt, p.t_final, p.max_steps)


def test_quad4_traction_closed_form():
    p = meshgen.hex8_cantilever(2, 2, 2, lx=2.0, ly=1.0, lz=3.0)
    face = rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 2.0))
    F = rio.traction_forces(p.coords, face, [0.7, 0.0, 9.0]).sum(axis=0)
    # normal = (dv x du)/|.| with the faces in the element's outward corner order (counter-
    # clockwise seen from outside): dv x du points into the body, here -x; s2 is not used
    assert np.allclose(F, [-0.7 * 3.0, 0.0, 0.0], rtol=1e-13, atol=1e-13)
    # tangential part: s1 du with du = dx/dxi1 not normalised (half the face edge per face)
    for fc in face:
        X = p.coords[fc]
        du = (X[1] - X[0]) / 2.0
        Ff = rio.traction_forces(p.coords, [fc], [0.0, 2.0, 0.0]).sum(axis=0)
        area = np.linalg.norm(np.cross(X[1] - X[0], X[3] - X[0]))
        assert np.allclose(Ff, 2.0 * du * area, rtol=1e-13)


def test_traction_matches_consistent_nodal_forces():
    """The cantilever's load, t = (0, 0, -0.05) on x = 4, given as a Tractions block with the
    faces ordered so that dx/dxi1 runs along z: identical nodal forces."""
    p = meshgen.hex8_cantilever(4, 2, 2)
    faces = [[fc[0], fc[3], fc[2], fc[1]] for fc in rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 4.0))]
    hz = 1.0 / 2
    F = rio.traction_forces(p.coords, faces, [0.0, -0.05 / (hz / 2.0), 0.0])
    assert np.allclose(F.ravel(), p.fnodal, rtol=1e-13, atol=1e-16)


def test_tri6_face_area_and_normal():
    X = np.array([[0, 0, 0], [2, 0, 0], [0, 3, 0], [1, 0, 0], [1, 1.5, 0], [0, 1.5, 0]], dtype=float)
    F = rio.traction_forces(X, [[0, 1, 2, 3, 4, 5]], [1.0, 0.0, 0.0])
    assert np.allclose(F.sum(axis=0), [0, 0, -3.0], rtol=1e-13)   # area 3, normal dv x du = -z
    assert np.allclose(F[:3].sum(axis=0), 0.0, atol=1e-13)         # vertex shares vanish for tri6


CONFIG = """
Files
{
  mesh : m.msh
}

Domains
{
  phase0
  {
    Material   : 2
    Element    : 1
  }
}

! a comment line
Material
{
  id : 2
  name : Matl_NeoHookean
  density : 1.0
  data_deviatoric :  3.5
  data_volumetric :  3  0.02
}

Boundary Conditions
{
    clamp
    {
        type   :  specified
        dof    :  X
        value  :  0.0
    }
}

Nodal Forces
{
  timefunction 1
  count 1
  9 3 -1.5
}

Time Functions
{
   1   0.0   1000.0  0.0  2.0    0.0   0.0   0.0   0.0   0.0   0.0
}

Solver
{
finalTime          1.0
timeStep           0.25
maximumSteps       4
maximumIterations  12
tolerance          1.0e-9
}
"""


def test_config_reader_rules(tmp_path):
    p = meshgen.hex8_cantilever(2, 1, 1)
    clamp = rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 0.0))
    rio.write_gmsh22(tmp_path / "m.msh", p, {"clamp": clamp})
    (tmp_path / "config").write_text(CONFIG)
    q = rio.read_config(tmp_path / "config")
    assert np.allclose(q.mats, [[3.5, 0.02, 3.0]])
    fx = q.fixed.reshape(-1, 3)
    clamped = np.isclose(p.coords[:, 0], 0.0)
    assert (fx[clamped, 0] == 1).all() and (fx[:, 1:] == 0).all() and (fx[~clamped] == 0).all()
    F = q.fnodal.reshape(-1, 3)
    assert F[8, 2] == -3.0 and np.count_nonzero(F) == 1          # lam = 2 t: the slope scales the load
    assert (q.dt, q.t_final, q.max_steps) == (0.25, 1.0, 4)
    assert q.meta["tolerance"] == 1e-9 and q.meta["maximumIterations"] == 12
    (tmp_path / "config").write_text(CONFIG.replace("0.0  2.0    0.0   0.0", "1.0  0.0    0.0   0.0"))
    with pytest.raises(NotImplementedError):
        rio.read_config(tmp_path / "config")                     # constant load: not lam = c t
    (tmp_path / "config").write_text(CONFIG.replace("value  :  0.0", "value  :  0.1"))
    q = rio.read_config(tmp_path / "config")                     # a nonzero value without a time
    assert np.all(q.presc_const.reshape(-1, 3)[clamped, 0] == 0.1)  # function: applied from the start
    assert not q.presc_ramp.any()
    (tmp_path / "config").write_text(CONFIG.replace("value  :  0.0", "value  :  0.1\n    timefunction : 1"))
    q = rio.read_config(tmp_path / "config")                     # with lam = 2 t: ramped
    assert np.all(q.presc_ramp.reshape(-1, 3)[clamped, 0] == 0.2) and not q.presc_const.any()
    (tmp_path / "config").write_text(CONFIG.replace("Matl_NeoHookean", "Matl_LinearElastic"))
    with pytest.raises(NotImplementedError):
        rio.read_config(tmp_path / "config")
    (tmp_path / "config").write_text(CONFIG.replace("Solver", "Solvr"))
    with pytest.raises(ValueError):
        rio.read_config(tmp_path / "config")                     # unknown block key


def test_material_models_round_trip(tmp_path):
    # Matl_MooneyRivlin / Matl_Gent read data_deviatoric; Matl_ArrudaBoyce reads its data line
    p = meshgen.two_phase_inclusions(16, 4, 4, seed=3, r_range=(0.2, 0.3))
    n_mat = len(p.mats)
    p.mat_model = np.array([1, 3][:n_mat], np.int32)
    p.mat_data = np.array([[0.4, 0.15, 0, 0], [0.7, 5.0, 0, 0]][:n_mat])
    p.mats[:, 0] = p.mat_data[:, 0]
    clamp = rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 0.0))
    q = _write(tmp_path, p, {"clamp": clamp})
    text = (tmp_path / "config").read_text()
    assert "Matl_MooneyRivlin" in text and "data_deviatoric : 0.4 0.15" in text
    assert "Matl_ArrudaBoyce" in text and "data            : 0.7 5.0" in text
    assert np.array_equal(q.mat_model[q.mat_id], p.mat_model[p.mat_id])
    assert np.array_equal(q.mat_data[q.mat_id], p.mat_data[p.mat_id])
    assert np.array_equal(q.mats[q.mat_id], p.mats[p.mat_id])


def test_gent_block(tmp_path):
    p = meshgen.hex8_cantilever(2, 1, 1)
    clamp = rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 0.0))
    rio.write_gmsh22(tmp_path / "m.msh", p, {"clamp": clamp})
    (tmp_path / "config").write_text(CONFIG.replace("Matl_NeoHookean", "Matl_Gent")
                                     .replace("data_deviatoric :  3.5", "data_deviatoric :  3.5 40.0"))
    q = rio.read_config(tmp_path / "config")
    assert q.mat_model.tolist() == [2] and np.allclose(q.mat_data, [[3.5, 40.0, 0, 0]])
    (tmp_path / "config").write_text(CONFIG.replace("Matl_NeoHookean", "Matl_Gent"))
    with pytest.raises(ValueError):
        rio.read_config(tmp_path / "config")                     # Gent needs mu and Im


EXAMPLE4 = "/root/reference/doc/examples/SolidMechanics/Example4/example4.rst"


def _example4_config():
    """The config of the reference's 3D mixed example (block under compression, Taylor-Hood
    ELEM_SOLID_3D_MIXED1): the literal block of its documentation page."""
    if not os.path.exists(EXAMPLE4):
        pytest.skip("the reference's documentation is not available here")
    lines = open(EXAMPLE4).read().splitlines()
    start = next(i for i, ln in enumerate(lines) if ln.rstrip().endswith("::")) + 1
    body = []
    for ln in lines[start:]:
        if ln.strip() and not ln.startswith(" "):
            break
        body.append(ln[4:] if ln.startswith("    ") else ln.strip())
    return "\n".join(body)


def test_reference_example4_config_parses():
    cfg = rio.parse_config(_example4_config())
    assert cfg["files"]["mesh"] == "block3d-P2-nelem8"
    assert cfg["elements"][0]["type"] == "ELEM_SOLID_3D_MIXED1"
    mat = cfg["materials"][0]
    assert mat["name"] == "Matl_NeoHookean"
    ut, kinv = mat["data_volumetric"].split()
    assert int(ut) == 3 and float(kinv) == pytest.approx(2.494128406043830e-06)
    assert float(mat["data_deviatoric"]) == pytest.approx(80.19367957863858)
    assert cfg["domains"]["block"] == (0, 0)
    assert cfg["tractions"]["pressure"]["value"].split() == ["-320", "0.0", "0.0"]
    s = cfg["solver"]
    assert (s["timeStep"], s["finalTime"], s["maximumSteps"], s["maximumIterations"]) == (0.2, 1.0, 10, 20)
    assert s["tolerance"] == pytest.approx(1e-7)
    assert cfg["tfs"][0](0.4) == pytest.approx(0.4)


def test_reference_example4_on_a_generated_block(tmp_path):
    """The example's config on a tet10 unit block with its patches (the quarter of the top face
    at x, y <= 1/2 loaded, the rest of the top held in x and y, symmetry planes): element type,
    material, the specified (zero) DOFs -- the config gives `top` and `pressure` one entry per DOF,
    and every entry counts -- and the load resultant 320 * 1/4 along z."""
    text = _example4_config()
    p = meshgen.tet10_kuhn(4, 4, 4, lx=1.0, jitter=0.0)
    X = p.coords
    on = lambda c, v: np.isclose(X[:, c], v)  # noqa: E731
    quarter = lambda Y: np.isclose(Y[:, 2], 1.0) & (Y[:, 0] <= 0.5 + 1e-12) & (Y[:, 1] <= 0.5 + 1e-12)  # noqa: E731
    pressure = rio.boundary_faces(p, quarter)
    top_all = rio.boundary_faces(p, lambda Y: np.isclose(Y[:, 2], 1.0))
    pk = {tuple(sorted(f)) for f in pressure}
    patches = {"symX": rio.boundary_faces(p, lambda Y: np.isclose(Y[:, 0], 0.0)),
               "symY": rio.boundary_faces(p, lambda Y: np.isclose(Y[:, 1], 0.0)),
               "symZ": rio.boundary_faces(p, lambda Y: np.isclose(Y[:, 2], 0.0)),
               "top": [f for f in top_all if tuple(sorted(f)) not in pk], "pressure": pressure}
    rio.write_gmsh22(tmp_path / "block.msh", p, patches, domain_names=["block"])
    (tmp_path / "example4.cfg").write_text(text)
    q = rio.read_config(tmp_path / "example4.cfg", mesh_path=tmp_path / "block.msh")
    assert q.meta["element"] == "ELEM_SOLID_3D_MIXED1"
    assert q.mats[0] == pytest.approx([80.19367957863858, 2.494128406043830e-06, 3.0])
    fx = q.fixed.reshape(-1, 3)
    assert np.all(fx[on(0, 0.0), 0] == 1) and np.all(fx[on(1, 0.0), 1] == 1) and np.all(fx[on(2, 0.0), 2] == 1)
    top = on(2, 1.0)
    assert np.all(fx[top, 0] == 1) and np.all(fx[top, 1] == 1)
    free_inside = ~(on(0, 0.0) | on(1, 0.0) | on(2, 0.0) | top)
    assert np.all(fx[free_inside] == 0)
    # the reference's face normal is dx/deta x dx/dxi (BasisFunctionsLagrange.cpp:1711), which points
    # into the block for the outward-ordered faces boundary_faces writes: s0 = -320 then pulls
    F = q.fnodal.reshape(-1, 3)
    assert F[:, 2].sum() == pytest.approx(320.0 * 0.25, rel=1e-12)
    assert np.abs(F[:, :2]).max() <= 1e-12 * 320
    assert (q.dt, q.t_final, q.max_steps) == (0.2, 1.0, 10)


def test_hex27_round_trip_and_element_type(tmp_path):
    """A 27-node hex mesh (Gmsh type 12, the same node order as the reference's hex27) with its
    quad9 clamp faces: read back as the same problem, element type ELEM_SOLID_3D_MIXED1."""
    p = meshgen.hex27_cantilever(3, 2, 2, jitter=0.1)
    clamp = rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 0.0))
    assert len(clamp) == 4 and all(len(fc) == 9 for fc in clamp)
    q = _write(tmp_path, p, {"clamp": clamp})
    assert q.npe == 27 and q.meta["element"] == "ELEM_SOLID_3D_MIXED1"
    assert np.array_equal(q.coords, p.coords) and np.array_equal(q.conn, p.conn)
    assert np.array_equal(q.fixed, p.fixed) and np.array_equal(q.fnodal, p.fnodal)


def test_quad9_traction_matches_consistent_nodal_forces():
    """The hex27 cantilever's load, t = (0, 0, -0.05) on x = 4, as a Tractions block on the quad9
    faces ordered so that dx/dxi1 runs along z: the generator's consistent nodal forces (the 1D
    quadratic weights 1/6, 2/3, 1/6, tensored), and the total force."""
    p = meshgen.hex27_cantilever(4, 2, 2, traction=(0.0, 0.0, -0.05))
    faces = [[fc[0], fc[3], fc[2], fc[1], fc[7], fc[6], fc[5], fc[4], fc[8]]
             for fc in rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 4.0))]
    hz = 1.0 / 2
    F = rio.traction_forces(p.coords, faces, [0.0, -0.05 / (hz / 2.0), 0.0])
    assert np.allclose(F.ravel(), p.fnodal, rtol=1e-13, atol=1e-16)
    assert np.allclose(F.sum(axis=0), [0.0, 0.0, -0.05 * 1.0], rtol=1e-13)
    # normal part: the face area (outward corner order: dv x du points into the body)
    Fn = rio.traction_forces(p.coords, rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 4.0)), [0.3, 0.0, 0.0])
    assert np.allclose(Fn.sum(axis=0), [-0.3, 0.0, 0.0], rtol=1e-13, atol=1e-15)


def test_prism18_is_refused_like_the_reference(tmp_path):
    """An 18-node prism mesh (Gmsh type 13) for ELEM_SOLID_3D_MIXED1: the reference declares the
    element (Elem_Solid_3D_Mixed1.cpp:48-53) but throws when it evaluates it (no ELEM_SHAPE_WEDGE
    branch in GeomDataLagrange.cpp:349-382, no 18-node case in LagrangeBasisFunsPrism), so the
    reader refuses the mesh."""
    p = meshgen.hex27_cantilever(2, 1, 1)
    clamp = rio.boundary_faces(p, lambda X: np.isclose(X[:, 0], 0.0))
    _write(tmp_path, p, {"clamp": clamp})
    lines = (tmp_path / "m.msh").read_text().splitlines()
    out = []
    for ln in lines:
        tok = ln.split()
        if len(tok) == 5 + 27 and tok[1] == "12":
            ln = " ".join([tok[0], "13"] + tok[2:5] + tok[5:23])
        out.append(ln)
    (tmp_path / "m.msh").write_text("\n".join(out) + "\n")
    with pytest.raises(NotImplementedError, match="18-node prisms"):
        rio.read_config(tmp_path / "config")

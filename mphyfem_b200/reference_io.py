"""The reference's input formats for the 3D solid path: Gmsh 2.2 meshes and the block-structured
``config`` file, read into a :class:`meshgen.Problem` (and written from one).

Restated behaviour (host-side, as in the reference):

* mesh: ``femBase::readInputGMSH`` (src/utilities/femBase.cpp:121-367). The highest physical
  dimension names the domains; every other physical name is a boundary patch. A mesh element
  line carries exactly two tags (``npElem = ntokens - 5``); the first tag is the physical tag.
  Node numbers are 1-based in the file, 0-based here.
* config: ``femBase::readInput`` (femBase.cpp:370-477) dispatches on the block keywords
  ``Files``, ``Model Type``, ``Domains``, ``Element``, ``Material``, ``Body Force``,
  ``Time Functions``, ``Solver``, ``Boundary Conditions``, ``Tractions``, ``Nodal Forces``,
  ``Output``, ``Nodal Data Output``; lines starting with ``!``, ``#`` or ``%`` are comments.
  ``Domains`` (Domain.cpp:32-72): per domain label ``Material : id`` and ``Element : id``
  (1-based). ``Material`` (MaterialBase.cpp:91-116; names of myIDmaps.h:233-236, objects of
  NewMaterial.h:48-54): ``Matl_NeoHookean`` (``data_deviatoric : mu``), ``Matl_MooneyRivlin``
  (``data_deviatoric : c1 c2``), ``Matl_Gent`` (``data_deviatoric : mu Im``) and
  ``Matl_ArrudaBoyce`` (``data : mu N``, the line its computeStressAndTangent reads,
  Matl_ArrudaBoyce.cpp:28), each with ``data_volumetric : Utype Kinv``. ``Boundary Conditions``
  (femBase.cpp:670-771, femSolidmechanics1.cpp:813-915): ``type : fixed`` prescribes every DOF
  of the patch's nodes to zero; ``type : specified`` prescribes ``dof`` to ``value``.
  ``Nodal Forces`` (femBase.cpp:876-919): ``timefunction n``, ``count m``, then m lines
  ``node dof value`` (1-based). ``Tractions`` (femBase.cpp:774-873): ``type : traction``,
  ``value : s0 s1 s2``, ``timefunction : n``. ``Time Functions`` (TimeFunction.cpp:47-68): lines
  ``id t0 t1 p1 .. p8``, lam(t) = p1 + p2 (t-t0) + p3 sin(p4 (t-t0) + p5) + p6 cos(p7 (t-t0) + p8)
  summed over the blocks with t0 <= t <= t1. ``Solver`` (femBase.cpp:994-1130): ``timeStep``,
  ``finalTime``, ``maximumSteps``, ``maximumIterations``, ``tolerance``.
* tractions: ``femSolidmechanics::addExternalForces`` (femSolidmechanics1.cpp:922-1119) on the
  reference geometry: at every face Gauss point, with du = dx/dxi1, dv = dx/dxi2,
  normal = (dv x du) / |dv x du|, dA = w |dv x du|, traction = (s0 normal + s1 du) dA (s2 is
  not used, du is not normalised); faces quad4 (4-point rule), tri3 (1 point), tri6 (3 points)
  with the shape functions of BasisFunctionsLagrange.cpp:296-700 and the rules of
  QuadratureUtil.cpp:360-600.

Limits of this build's Newton driver, checked with clear errors: the load factor must be
proportional to time (lam(t) = c t on [0, finalTime]: the driver steps lam = t and the forces are
scaled by c); prescribed values must be zero; no body force; the four hyperelastic materials
above; hex8 or tet10 volumes. The ``Solver`` block also accepts ``key value`` lines without the colon, the
form the reference's own sample config uses (its reader splits on ``:`` only).
"""
from __future__ import annotations

import math

import numpy as np

from .meshgen import Problem

GMSH_VOLUME = {5: 8, 11: 10, 12: 27}  # hex8, tet10, hex27 (the 27-node hex order is Gmsh's)
GMSH_PRISM18 = 13
# material name -> (model code of mphy.h, config line holding its parameters, parameter count)
MATERIALS = {"Matl_NeoHookean": (0, "data_deviatoric", 1), "Matl_MooneyRivlin": (1, "data_deviatoric", 2),
             "Matl_Gent": (2, "data_deviatoric", 2), "Matl_ArrudaBoyce": (3, "data", 2)}
MATERIAL_NAME = {code: name for name, (code, _, _) in MATERIALS.items()}
GMSH_FACE = {3: 4, 2: 3, 9: 6, 10: 9}  # quad4, tri3, tri6, quad9
GMSH_TYPE_OF = {8: 5, 10: 11, 27: 12, 4: 3, 3: 2, 6: 9, 9: 10}
DOF_NAMES = {"x": 0, "y": 1, "z": 2, "ux": 0, "uy": 1, "uz": 2, "0": 0, "1": 1, "2": 2}


# ----------------------------------------------------------------------------------- Gmsh 2.2
def read_gmsh22(path):
    """Returns dict(nodes [n, 3], domains {name: tag}, patches {name: tag},
    volume [(type, tag, nodes0)], faces {patch name: [nodes0, ...]})."""
    with open(path) as f:
        lines = [ln.strip() for ln in f]
    i = 0

    def expect(tok):
        nonlocal i
        while i < len(lines) and not lines[i]:
            i += 1
        if lines[i] != tok:
            raise ValueError(f"{path}: expected {tok}, found {lines[i]!r}")
        i += 1

    expect("$MeshFormat")
    version = lines[i].split()[0]
    if not version.startswith("2"):
        raise ValueError(f"{path}: Gmsh format {version}, expected 2.2 ASCII")
    i += 1
    expect("$EndMeshFormat")
    expect("$PhysicalNames")
    nphys = int(lines[i])
    i += 1
    phys = []
    for _ in range(nphys):
        dim, tag, name = lines[i].split(maxsplit=2)
        phys.append((int(dim), int(tag), name.strip().strip('"')))
        i += 1
    expect("$EndPhysicalNames")
    ndim = max(p[0] for p in phys)
    if ndim == 1:
        ndim = 2
    domains = {name: tag for dim, tag, name in phys if dim == ndim}
    patches = {name: tag for dim, tag, name in phys if dim < ndim}
    expect("$Nodes")
    nn = int(lines[i])
    i += 1
    nodes = np.zeros((nn, 3))
    for k in range(nn):
        t = lines[i].split()
        if int(t[0]) != k + 1:
            raise ValueError(f"{path}: node numbers must be 1..{nn} in order")
        nodes[k] = [float(t[1]), float(t[2]), float(t[3])]
        i += 1
    expect("$EndNodes")
    expect("$Elements")
    ne = int(lines[i])
    i += 1
    dom_tags = set(domains.values())
    tag_patch = {tag: name for name, tag in patches.items()}
    volume, faces = [], {name: [] for name in patches}
    for _ in range(ne):
        t = [int(x) for x in lines[i].split()]
        i += 1
        if t[2] != 2:
            raise ValueError(f"{path}: element lines must carry exactly 2 tags (femBase.cpp:284-327)")
        etype, tag, conn = t[1], t[3], [x - 1 for x in t[5:]]
        if tag in dom_tags:
            volume.append((etype, tag, conn))
        elif tag in tag_patch:
            faces[tag_patch[tag]].append(conn)
        else:
            raise ValueError(f"{path}: element with undeclared physical tag {tag}")
    expect("$EndElements")
    return dict(ndim=ndim, nodes=nodes, domains=domains, patches=patches, volume=volume, faces=faces)


def write_gmsh22(path, prob: Problem, patches: dict, domain_names=None):
    """Mesh of `prob` with its volume elements (physical tag = material index + 1, one domain per
    material) and boundary patches {name: [face node lists (0-based)]}."""
    nmat = len(prob.mats)
    domain_names = domain_names or [f"phase{m}" for m in range(nmat)]
    ptag = {name: nmat + 1 + k for k, name in enumerate(patches)}
    with open(path, "w") as f:
        f.write("$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$PhysicalNames\n")
        f.write(f"{nmat + len(patches)}\n")
        for name, tag in ptag.items():
            f.write(f'2 {tag} "{name}"\n')
        for m in range(nmat):
            f.write(f'3 {m + 1} "{domain_names[m]}"\n')
        f.write("$EndPhysicalNames\n$Nodes\n")
        f.write(f"{prob.n_node}\n")
        for k, (x, y, z) in enumerate(prob.coords):
            f.write(f"{k + 1} {float(x)!r} {float(y)!r} {float(z)!r}\n")
        f.write("$EndNodes\n$Elements\n")
        nf = sum(len(v) for v in patches.values())
        f.write(f"{nf + prob.n_elem}\n")
        k = 1
        for name, flist in patches.items():
            for fc in flist:
                f.write(f"{k} {GMSH_TYPE_OF[len(fc)]} 2 {ptag[name]} {ptag[name]} " + " ".join(str(v + 1) for v in fc)
                        + "\n")
                k += 1
        et = GMSH_TYPE_OF[prob.npe]
        for e in range(prob.n_elem):
            tag = int(prob.mat_id[e]) + 1
            f.write(f"{k} {et} 2 {tag} {tag} " + " ".join(str(v + 1) for v in prob.conn[e]) + "\n")
            k += 1
        f.write("$EndElements\n")


# ----------------------------------------------------------------------------------- config
def _active(line):
    return len(line) > 0 and line[0] not in "!#%"


def _blocks(text):
    """Top-level (keyword, body lines) pairs; nested blocks stay inside the body."""
    lines = [ln.strip() for ln in text.splitlines()]
    out, i = [], 0
    while i < len(lines):
        ln = lines[i]
        i += 1
        if not _active(ln) or ln in ("{", "}"):
            continue
        while i < len(lines) and not _active(lines[i]):
            i += 1
        if i >= len(lines) or lines[i] != "{":
            raise ValueError(f"config: block {ln!r} without '{{'")
        depth, body, i = 1, [], i + 1
        while i < len(lines) and depth:
            s = lines[i]
            i += 1
            if s.startswith("{"):
                depth += 1
            elif s.startswith("}"):
                depth -= 1
                if depth == 0:
                    break
            body.append(s)
        out.append((ln, body))
    return out


def _kv(line):
    if ":" in line:
        k, v = line.split(":", 1)
    else:
        parts = line.split(None, 1)
        k, v = parts[0], (parts[1] if len(parts) > 1 else "")
    return k.strip(), v.strip()


def _sub_blocks(body):
    """label { key : value ... } entries inside a block body -> {label: {key: value}} (a label
    given twice keeps its last entry; see _sub_block_list for blocks that repeat labels)."""
    return dict(_sub_block_list(body))


def _sub_block_list(body):
    """label { key : value ... } entries inside a block body, in order, as (label, {key: value}):
    the reference reads every entry, so one patch may carry several entries (one per DOF)."""
    out, i = [], 0
    while i < len(body):
        ln = body[i]
        i += 1
        if not _active(ln) or ln in ("{", "}"):
            continue
        label = ln
        while i < len(body) and body[i] != "{":
            i += 1
        i += 1
        kv = {}
        while i < len(body) and not body[i].startswith("}"):
            if _active(body[i]):
                k, v = _kv(body[i])
                kv[k] = v
            i += 1
        i += 1
        out.append((label, kv))
    return out


class TimeFunction:
    """lam(t) of TimeFunction.cpp:47-68 (sum over blocks with t0 <= t <= t1, tolerance 1e-12)."""

    def __init__(self):
        self.blocks = []

    def __call__(self, t):
        lam = 0.0
        for t0, t1, p in self.blocks:
            if t < t0 - 1e-12 or t > t1 - 1e-12:
                continue
            d = t - t0
            lam += p[0] + p[1] * d + p[2] * math.sin(p[3] * d + p[4]) + p[5] * math.cos(p[6] * d + p[7])
        return lam


# shape functions of the boundary faces (the reference's node orders) and their rules
_G = 0.577350269189626


_G3 = (-0.774596669241483, 0.774596669241483, 0.0)   # QuadratureUtil.cpp:29-33
_W3 = (5.0 / 9.0, 5.0 / 9.0, 8.0 / 9.0)


def _face_rule(npf):
    if npf == 4:
        return [(-_G, -_G, 1.0), (_G, -_G, 1.0), (_G, _G, 1.0), (-_G, _G, 1.0)]
    if npf == 9:
        # 3x3 rule on the quad9 face (its points in xi1-fastest order)
        return [(_G3[i], _G3[j], _W3[i] * _W3[j]) for j in range(3) for i in range(3)]
    if npf == 3:
        return [(1.0 / 3.0, 1.0 / 3.0, 0.5)]
    if npf == 6:
        return [(1.0 / 6.0, 1.0 / 6.0, 0.5 / 3.0), (4.0 / 6.0, 1.0 / 6.0, 0.5 / 3.0), (1.0 / 6.0, 4.0 / 6.0, 0.5 / 3.0)]
    raise ValueError(f"face with {npf} nodes: quad4, quad9, tri3 and tri6 faces are supported")


# quad9 face nodes (BasisFunctionsLagrange.cpp, LagrangeBasisFunsQuad case 9): the 1D quadratic
# indices (u, v) of each node, 0 at -1, 1 at +1, 2 at the midpoint -- corners, mid-edges of
# (0,1), (1,2), (2,3), (3,0), centre (Gmsh's quad9 order)
_QUAD9 = ((0, 0), (1, 0), (1, 1), (0, 1), (2, 0), (1, 2), (2, 1), (0, 2), (2, 2))


def _face_shape(npf, a, b):
    if npf == 9:
        def q(x):
            return (0.5 * (x * x - x), 0.5 * (x * x + x), 1.0 - x * x), (x - 0.5, x + 0.5, -2.0 * x)
        nu, dnu = q(a)
        nv, dnv = q(b)
        N = np.array([nv[j] * nu[i] for i, j in _QUAD9])
        d1 = np.array([nv[j] * dnu[i] for i, j in _QUAD9])
        d2 = np.array([dnv[j] * nu[i] for i, j in _QUAD9])
        return N, d1, d2
    if npf == 4:
        nu, dnu = [0.5 * (1 - a), 0.5 * (1 + a)], [-0.5, 0.5]
        nv, dnv = [0.5 * (1 - b), 0.5 * (1 + b)], [-0.5, 0.5]
        order = [(0, 0), (1, 0), (1, 1), (0, 1)]  # N0 = v0 u0, N1 = v0 u1, N2 = v1 u1, N3 = v1 u0
        N = np.array([nv[j] * nu[i] for i, j in order])
        d1 = np.array([nv[j] * dnu[i] for i, j in order])
        d2 = np.array([dnv[j] * nu[i] for i, j in order])
        return N, d1, d2
    c = 1.0 - a - b
    if npf == 3:
        return np.array([c, a, b]), np.array([-1.0, 1.0, 0.0]), np.array([-1.0, 0.0, 1.0])
    N = np.array([c * (2 * c - 1), a * (2 * a - 1), b * (2 * b - 1), 4 * a * c, 4 * a * b, 4 * b * c])
    d1 = np.array([-(4 * c - 1), 4 * a - 1, 0.0, 4 * (c - a), 4 * b, -4 * b])
    d2 = np.array([-(4 * c - 1), 0.0, 4 * b - 1, -4 * a, 4 * a, 4 * (c - b)])
    return N, d1, d2


def traction_forces(coords, faces, value):
    """Consistent nodal forces [n_node, 3] of a traction (s0 normal + s1 dx/dxi1) on the faces,
    femSolidmechanics1.cpp:1013-1067."""
    F = np.zeros((len(coords), 3))
    s0, s1 = float(value[0]), float(value[1])
    for fc in faces:
        fc = np.asarray(fc)
        X = coords[fc]
        for a, b, w in _face_rule(len(fc)):
            N, d1, d2 = _face_shape(len(fc), a, b)
            du, dv = d1 @ X, d2 @ X
            nrm = np.cross(dv, du)
            jac = np.linalg.norm(nrm)
            t = (s0 * nrm / jac + s1 * du) * (w * jac)
            F[fc] += N[:, None] * t[None, :]
    return F


# element types of the reference's Element block (myIDmaps.h) that this build solves
ELEMENT_TYPES = ("ELEM_SOLID_3D_DISP", "ELEM_SOLID_3D_MIXED0", "ELEM_SOLID_3D_MIXED1")


def parse_config(text):
    """The blocks of a reference config (femBase::readInput, femBase.cpp:121-364): a dict with
    files, domains {label: (material, element)}, materials {id: {key: value}}, elements
    {id: {key: value}}, bcs, tractions {patch: {key: value}}, tfs {id: TimeFunction}, nodal
    (time function, [(node, dof, value)]) or None, and solver {timeStep, finalTime, maximumSteps,
    maximumIterations, tolerance}. Ids are 0-based."""
    blocks = _blocks(text)
    files, domains, materials, elements, bcs, tractions, tfs = {}, {}, {}, {}, [], {}, {}
    nodal = None
    solver = dict(timeStep=1.0, finalTime=1.0, maximumSteps=1, maximumIterations=10, tolerance=1e-10)
    for key, body in blocks:
        if key == "Files":
            for ln in body:
                if _active(ln):
                    k, v = _kv(ln)
                    files[k] = v
        elif key == "Domains":
            for label, kv in _sub_blocks(body).items():
                domains[label] = (int(kv["Material"]) - 1, int(kv.get("Element", "1")) - 1)
        elif key == "Material":
            kv = dict(_kv(ln) for ln in body if _active(ln))
            materials[int(kv["id"]) - 1] = kv
        elif key == "Element":
            kv = dict(_kv(ln) for ln in body if _active(ln))
            elements[int(kv["id"]) - 1] = kv
        elif key == "Body Force":
            kv = dict(_kv(ln) for ln in body if _active(ln))
            if any(float(x) != 0.0 for x in kv.get("value", "0").split()):
                raise NotImplementedError("config: a nonzero body force is not supported by this build")
        elif key == "Boundary Conditions":
            bcs = _sub_block_list(body)
        elif key == "Tractions":
            tractions = _sub_blocks(body)
        elif key == "Nodal Forces":
            act = [ln for ln in body if _active(ln)]
            tf = int(act[0].split()[1]) - 1
            count = int(act[1].split()[1])
            data = [(int(a) - 1, int(b) - 1, float(c)) for a, b, c in (ln.split() for ln in act[2:2 + count])]
            nodal = (tf, data)
        elif key == "Time Functions":
            for ln in body:
                if not _active(ln):
                    continue
                v = [float(x) for x in ln.split()]
                tfs.setdefault(int(v[0]) - 1, TimeFunction()).blocks.append((v[1], v[2], v[3:11]))
        elif key == "Solver":
            for ln in body:
                if not _active(ln):
                    continue
                k, v = _kv(ln)
                if k == "timeStep":
                    solver[k] = float(v.split()[0])
                elif k in ("finalTime", "tolerance"):
                    solver[k] = float(v)
                elif k in ("maximumSteps", "maximumIterations"):
                    solver[k] = int(v)
        elif key in ("Model Type", "Output", "Nodal Data Output"):
            continue
        else:
            raise ValueError(f"config: key not found: {key!r} (femBase::readInput)")
    return dict(files=files, domains=domains, materials=materials, elements=elements, bcs=bcs, tractions=tractions,
                tfs=tfs, nodal=nodal, solver=solver)


def read_config(config_path, mesh_path=None):
    """A Problem from the reference's config (and the mesh it names, relative to the config's
    directory, unless mesh_path is given). meta carries the Solver block's tolerance and
    maximumIterations, the domains, and the element type of the domains' Element block."""
    import os
    cfg = parse_config(open(config_path).read())
    files, domains, materials, elements = cfg["files"], cfg["domains"], cfg["materials"], cfg["elements"]
    bcs, tractions, tfs, nodal, solver = cfg["bcs"], cfg["tractions"], cfg["tfs"], cfg["nodal"], cfg["solver"]
    mesh_path = mesh_path or os.path.join(os.path.dirname(os.path.abspath(config_path)), files["mesh"])
    m = read_gmsh22(mesh_path)
    if m["ndim"] != 3:
        raise NotImplementedError("config: this build solves 3D meshes (hex8, tet10, hex27)")
    vol = m["volume"]
    if any(t == GMSH_PRISM18 for t, _, _ in vol):
        # Elem_Solid_3D_Mixed1 declares the 18-node wedge (Elem_Solid_3D_Mixed1.cpp:48-53), but the
        # reference cannot evaluate it: computeBasisFunctions3D has no branch for ELEM_SHAPE_WEDGE
        # and throws (GeomDataLagrange.cpp:349-382), and LagrangeBasisFunsPrism defines the 6-node
        # prism only (BasisFunctionsLagrange.cpp:1412-1490). The same refusal here.
        raise NotImplementedError("mesh: 18-node prisms (Gmsh type 13) have no Lagrange basis in the reference "
                                  "(computeBasisFunctions3D ... Invalid element type)")
    npe = {GMSH_VOLUME.get(t) for t, _, _ in vol}
    if None in npe or len(npe) != 1:
        raise NotImplementedError("mesh: volume elements must all be hex8 (type 5), all tet10 (type 11) or all "
                                  "hex27 (type 12)")
    npe = npe.pop()
    # materials: one row per material the domains use, in domain-tag order of first use
    tag_mat = {}
    for label, tag in m["domains"].items():
        if label not in domains:
            raise ValueError(f"config: domain {label!r} of the mesh has no Domains entry")
        tag_mat[tag] = domains[label][0]
    used = sorted(set(tag_mat.values()))
    rows, models, mdata = [], [], []
    for mid in used:
        kv = materials.get(mid)
        if kv is None:
            raise ValueError(f"config: material {mid + 1} is not defined")
        if kv.get("name") not in MATERIALS:
            raise NotImplementedError(f"config: material {kv.get('name')!r}: supported are {sorted(MATERIALS)}")
        code, line, npar = MATERIALS[kv["name"]]
        if line not in kv:
            raise ValueError(f"config: material {mid + 1} ({kv['name']}) has no {line} line")
        par = [float(x) for x in kv[line].split()]
        if len(par) < npar:
            raise ValueError(f"config: {kv['name']} needs {npar} values on its {line} line")
        ut, kinv = kv["data_volumetric"].split()[:2]
        rows.append([par[0], float(kinv), float(int(ut))])
        d = np.zeros(4)
        d[:npar] = par[:npar]
        models.append(code)
        mdata.append(d)
    row_of = {mid: k for k, mid in enumerate(used)}
    conn = np.array([c for _, _, c in vol], dtype=np.int32)
    mat_id = np.array([row_of[tag_mat[tag]] for _, tag, _ in vol], dtype=np.int32)
    coords = m["nodes"]
    n_node = len(coords)
    # loads at unit time, with lam(t) = slope t checked on the steps
    dt, tfin = solver["timeStep"], solver["finalTime"]
    ts = [dt * k for k in range(1, int(round(tfin / dt)) + 1)] or [dt]

    def slope_of(tf_index):
        if tf_index < 0:
            raise NotImplementedError("config: loads without a time function are constant; the driver ramps lam = t")
        fn = tfs[tf_index]
        c = fn(ts[0]) / ts[0]
        for t in ts:
            if abs(fn(t) - c * t) > 1e-12 * max(1.0, abs(c * t)):
                raise NotImplementedError("config: the load factor must be proportional to time (lam = c t)")
        return c

    # prescribed DOFs and their values
    fixed = np.zeros((n_node, 3), dtype=np.uint8)
    presc_ramp, presc_const = np.zeros((n_node, 3)), np.zeros((n_node, 3))
    for label, kv in bcs:
        if label not in m["faces"]:
            raise ValueError(f"config: boundary condition on unknown patch {label!r}")
        nodes = sorted({v for fc in m["faces"][label] for v in fc})
        if kv.get("type") == "fixed":
            fixed[nodes, :] = 1
        elif kv.get("type") == "specified":
            # value(t) = value * lam(t) with the entry's time function, or value from the first
            # step without one (femSolidmechanics1.cpp:840-868); constants only (no expressions)
            dof = DOF_NAMES[kv["dof"].strip().lower()]
            fixed[nodes, dof] = 1
            value = float(kv.get("value", "0"))
            if value != 0.0:
                tfn = int(kv.get("timefunction", "0")) - 1
                if tfn >= 0:
                    presc_ramp[nodes, dof] = slope_of(tfn) * value
                else:
                    presc_const[nodes, dof] = value
        else:
            raise ValueError(f"config: patch type {kv.get('type')!r} (femSolidmechanics::setBoundaryConditions)")
    F = np.zeros((n_node, 3))
    for label, kv in tractions.items():
        if kv.get("type") != "traction":
            raise ValueError(f"config: traction type {kv.get('type')!r}")
        c = slope_of(int(kv.get("timefunction", "0")) - 1)
        F += c * traction_forces(coords, m["faces"][label], [float(x) for x in kv["value"].split()])
    if nodal is not None:
        c = slope_of(nodal[0])
        for n, d, v in nodal[1]:
            F[n, d] += c * v
    etypes = {elements.get(domains[label][1], {}).get("type", "ELEM_SOLID_3D_DISP") for label in m["domains"]}
    if len(etypes) != 1:
        raise NotImplementedError("config: every domain must use the same element type")
    etype = etypes.pop()
    if etype not in ELEMENT_TYPES:
        raise NotImplementedError(f"config: element type {etype!r}: supported are {ELEMENT_TYPES}")
    if etype == "ELEM_SOLID_3D_MIXED1" and npe not in (10, 27):
        raise NotImplementedError("config: ELEM_SOLID_3D_MIXED1 is built for tet10 and hex27 meshes")
    if npe == 27 and etype != "ELEM_SOLID_3D_MIXED1":
        raise NotImplementedError("config: 27-node hexes are built for ELEM_SOLID_3D_MIXED1 (P2-P1) only")
    prob = Problem(name=os.path.basename(config_path), coords=coords, conn=conn, mat_id=mat_id,
                   mats=np.array(rows, dtype=np.float64), fixed=fixed.ravel(), fnodal=F.ravel(),
                   dt=dt, t_final=tfin, max_steps=solver["maximumSteps"],
                   meta={"tolerance": solver["tolerance"], "maximumIterations": solver["maximumIterations"],
                         "domains": m["domains"], "patches": list(m["patches"]), "element": etype})
    if presc_ramp.any() or presc_const.any():
        prob.presc_ramp, prob.presc_const = presc_ramp.ravel(), presc_const.ravel()
    if any(models):
        prob.mat_model = np.array(models, dtype=np.int32)
        prob.mat_data = np.array(mdata, dtype=np.float64)
    return prob


def write_config(path, mesh_name, prob: Problem, fixed_patches=(), domain_names=None, nodal_forces=True,
                 tractions=None):
    """A reference config for `prob`: one Material and Domain per material row, `fixed` patches,
    the nodal forces of `prob.fnodal` and the `tractions` {patch: (s0, s1, s2)}, both under time
    function 1 (lam = t), and its Solver settings."""
    nmat = len(prob.mats)
    domain_names = domain_names or [f"phase{m}" for m in range(nmat)]
    out = ["Files", "{", f"  mesh : {mesh_name}", "}", "", "Domains", "{"]
    for m in range(nmat):
        out += [f"  {domain_names[m]}", "  {", f"    Material : {m + 1}", "    Element  : 1", "  }"]
    out += ["}", ""]
    for m, (mu, kinv, ut) in enumerate(prob.mats):
        code = int(prob.mat_model[m]) if prob.mat_model is not None else 0
        name = MATERIAL_NAME[code]
        _, line, npar = MATERIALS[name]
        par = prob.mat_data[m][:npar] if prob.mat_model is not None else [mu]
        out += ["Material", "{", f"  id              : {m + 1}", f"  name            : {name}",
                "  density         : 1.0", f"  {line:<15} : " + " ".join(repr(float(v)) for v in par),
                f"  data_volumetric : {int(ut)} {float(kinv)!r}", "}", ""]
    etype = prob.meta.get("element") or ("ELEM_SOLID_3D_MIXED1" if prob.npe == 27 else "ELEM_SOLID_3D_DISP")
    if etype == "hex27":
        etype = "ELEM_SOLID_3D_MIXED1"
    out += ["Element", "{", "  id   : 1", f"  type : {etype}", "}", ""]
    if fixed_patches:
        out += ["Boundary Conditions", "{"]
        for name in fixed_patches:
            out += [f"  {name}", "  {", "    type : fixed", "  }"]
        out += ["}", ""]
    if tractions:
        out += ["Tractions", "{"]
        for name, val in tractions.items():
            out += [f"  {name}", "  {", "    type         : traction",
                    "    value        : " + " ".join(repr(float(v)) for v in val), "    timefunction : 1", "  }"]
        out += ["}", ""]
    if nodal_forces:
        F = prob.fnodal.reshape(-1, 3)
        nz = [(n, d, F[n, d]) for n in range(len(F)) for d in range(3) if F[n, d] != 0.0]
        out += ["Nodal Forces", "{", "  timefunction 1", f"  count {len(nz)}"]
        out += [f"  {n + 1} {d + 1} {float(v)!r}" for n, d, v in nz]
        out += ["}", ""]
    out += ["Time Functions", "{", "  1   0.0   1000.0   0.0  1.0   0.0  0.0  0.0   0.0  0.0  0.0", "}", "",
            "Solver", "{", "  solvertype        : newton", "  timescheme        : STEADY",
            f"  finalTime         : {float(prob.t_final)!r}", f"  timeStep          : {float(prob.dt)!r}",
            f"  maximumSteps      : {prob.max_steps}", "  maximumIterations : 10",
            f"  tolerance         : {float(prob.newton_rtol)!r}", "}", ""]
    with open(path, "w") as f:
        f.write("\n".join(out))


def boundary_faces(prob: Problem, predicate):
    """Faces of the volume elements whose nodes all satisfy predicate(coords) (hex8: quad4 faces
    in the element's outward corner order; hex27: quad9 faces, the same corners, then the
    mid-edge nodes and the face centre; tet10: tri6 faces), each face once."""
    if prob.npe == 8:
        local = [[0, 3, 2, 1], [4, 5, 6, 7], [0, 1, 5, 4], [1, 2, 6, 5], [2, 3, 7, 6], [3, 0, 4, 7]]
    elif prob.npe == 27:
        local = [[0, 3, 2, 1, 9, 13, 11, 8, 20], [4, 5, 6, 7, 16, 18, 19, 17, 25],
                 [0, 1, 5, 4, 8, 12, 16, 10, 21], [1, 2, 6, 5, 11, 14, 18, 12, 23],
                 [2, 3, 7, 6, 13, 15, 19, 14, 24], [3, 0, 4, 7, 9, 10, 17, 15, 22]]
    else:
        # tet10 faces: vertices then the mid-side nodes of (0,1), (1,2), (2,0) of the face
        local = [[0, 2, 1, 6, 5, 4], [0, 1, 3, 4, 9, 7], [1, 2, 3, 5, 8, 9], [0, 3, 2, 7, 8, 6]]
    ok = predicate(prob.coords)
    seen, out = set(), []
    for e in range(prob.n_elem):
        for lf in local:
            fc = [int(prob.conn[e, k]) for k in lf]
            if all(ok[fc]):
                key = tuple(sorted(fc))
                if key not in seen:
                    seen.add(key)
                    out.append(fc)
    return out


__all__ = ["read_gmsh22", "write_gmsh22", "read_config", "write_config", "traction_forces", "boundary_faces",
           "TimeFunction"]

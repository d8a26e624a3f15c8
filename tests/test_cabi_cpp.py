"""The C ABI from C++: tests/cabi_adapter.cpp drives libmphy.so through the SolverGpu adapter
(include/mphy_solver_gpu.hpp), the class a maintainer adds beside SolverPetsc.

CPU: the adapter and the driver compile with g++ against include/ alone (-Wall -Wextra -Werror),
and link against libmphy.so. GPU: the driver runs config 1 (hex8 32x8x8) twice -- the fused
GPU Newton iteration, and the reference's element-by-element assembleMatrixAndVector with the
oracle's element matrices -- and both solutions match the oracle's Jacobi-PCG solve to 1e-9.
"""
import os
import shutil
import subprocess

import numpy as np
import pytest

from mphyfem_b200 import build, meshgen

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "cabi_adapter.cpp")
LIBDIR = os.path.join(ROOT, "mphyfem_b200")
GXX = shutil.which("g++") or "/usr/bin/g++"
FLAGS = ["-std=c++17", "-O2", "-Wall", "-Wextra", "-Werror", "-I", os.path.join(ROOT, "include")]


def _link(out):
    build.build()
    cmd = [GXX, *FLAGS, SRC, "-L", LIBDIR, "-lmphy", f"-Wl,-rpath,{LIBDIR}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_adapter_compiles_against_the_header_alone():
    r = subprocess.run([GXX, *FLAGS, "-fsyntax-only", SRC], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    # the header on its own, as a reference translation unit would include it
    r = subprocess.run([GXX, *FLAGS, "-fsyntax-only", "-x", "c++", os.path.join(ROOT, "include",
                                                                                 "mphy_solver_gpu.hpp")],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]


def test_adapter_links_against_libmphy(tmp_path):
    _link(str(tmp_path / "cabi_adapter"))


def _write_input(path, p, oracle, lam):
    op = oracle.OracleProblem(p)
    _, fav, rp, _ = op.pattern()
    Ke, Fe, bad = op.elements(np.zeros(p.n_dof))
    assert bad == -1
    with open(path, "wb") as f:
        np.array([p.n_node, p.n_elem, p.npe, p.mats.shape[0], op.n_free], np.int32).tofile(f)
        np.ascontiguousarray(p.coords, np.float64).tofile(f)
        np.ascontiguousarray(p.conn, np.int32).tofile(f)
        np.ascontiguousarray(p.mat_id, np.int32).tofile(f)
        np.ascontiguousarray(p.mats, np.float64).tofile(f)
        np.ascontiguousarray(p.fixed, np.uint8).tofile(f)
        np.ascontiguousarray(p.fnodal, np.float64).tofile(f)
        np.array([lam], np.float64).tofile(f)
        np.diff(rp).astype(np.int32).tofile(f)
        np.ascontiguousarray(fav, np.int32).tofile(f)
        np.ascontiguousarray(Ke, np.float64).tofile(f)
        np.ascontiguousarray(Fe, np.float64).tofile(f)
    return op


@pytest.mark.gpu
def test_adapter_solves_config1_like_the_oracle(tmp_path, oracle):
    import torch
    if not torch.cuda.is_available():
        pytest.skip("no GPU")
    exe = str(tmp_path / "cabi_adapter")
    _link(exe)
    p = meshgen.cantilever_small()
    lam = 0.2
    op = _write_input(tmp_path / "in.bin", p, oracle, lam)
    r = subprocess.run([exe, str(tmp_path / "in.bin"), str(tmp_path / "out.bin")], capture_output=True, text=True,
                       timeout=300)
    assert r.returncode == 0, r.stdout[-2000:] + r.stderr[-2000:]
    raw = open(tmp_path / "out.bin", "rb").read()
    nd = p.n_dof
    du_fused = np.frombuffer(raw, np.float64, nd, 0)
    du_elem = np.frombuffer(raw, np.float64, nd, 8 * nd)
    norm_fused, norm_elem = np.frombuffer(raw, np.float64, 2, 16 * nd)
    its_fused, its_elem, status_before = np.frombuffer(raw, np.int32, 3, 16 * nd + 16)
    assert status_before == -1  # factoriseAndSolve before any assembly, as SolverPetsc
    # the oracle: assembled system at u = 0, rhs += lambda Fext, Jacobi-PCG to 1e-12
    val, rhs, _, _ = op.assemble(np.zeros(nd))
    free = np.flatnonzero(p.fixed == 0)
    b = rhs + lam * p.fnodal[free]
    x, its, _, st = op.cg(val, b, rtol=1e-12)
    assert st == 0
    assert norm_fused == pytest.approx(np.linalg.norm(b), rel=1e-12)
    assert norm_elem == pytest.approx(np.linalg.norm(b), rel=1e-12)
    for du, k in ((du_fused, its_fused), (du_elem, its_elem)):
        assert abs(int(k) - its) <= 2
        assert np.linalg.norm(du[free] - x) <= 1e-9 * np.linalg.norm(x)
        assert np.all(du[p.fixed == 1] == 0.0)

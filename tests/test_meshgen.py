"""Synthetic workload generators: sizes, loads, orientation, inclusion assignment."""
import numpy as np
import pytest

from mphyfem_b200 import meshgen


def test_cantilever_sizes_and_load():
    p = meshgen.cantilever_small()
    assert (p.n_node, p.n_elem, p.n_free) == (2673, 2048, 7776)
    # consistent nodal forces of t = (0, 0, -0.05) on the 1 x 1 end face
    assert p.fnodal.reshape(-1, 3).sum(axis=0) == pytest.approx([0.0, 0.0, -0.05], abs=1e-15)
    assert np.all(p.fixed.reshape(-1, 3)[np.isclose(p.coords[:, 0], 0.0)] == 1)
    assert p.fixed.sum() == 3 * 81


def test_large_config_counts():
    nx, ny, nz = 256, 64, 64
    assert (nx + 1) * (ny + 1) * (nz + 1) == 1085825
    assert 3 * (nx + 1) * (ny + 1) * (nz + 1) == 3257475


def test_tet10_orientation_midsides_and_load():
    p = meshgen.tet10_kuhn(4, 3, 3)
    v = p.coords[p.conn[:, :4]]
    vol = np.einsum("ij,ij->i", np.cross(v[:, 1] - v[:, 0], v[:, 2] - v[:, 0]), v[:, 3] - v[:, 0]) / 6
    assert np.all(vol > 0)
    assert vol.sum() == pytest.approx(4.0, rel=1e-12)
    for e, (a, b) in enumerate(meshgen.TET10_EDGES):
        mid = 0.5 * (p.coords[p.conn[:, a]] + p.coords[p.conn[:, b]])
        assert np.allclose(p.coords[p.conn[:, 4 + e]], mid)
    assert p.fnodal.reshape(-1, 3).sum(axis=0) == pytest.approx([0.0, 0.0, -0.02], abs=1e-14)


def test_two_phase_assignment_matches_brute_force():
    p = meshgen.two_phase_inclusions(20, 6, 5, seed=4, r_range=(0.12, 0.3))
    assert p.meta["vol_frac"] >= 0.2 and p.mats.shape == (2, 3)
    # recompute the sphere set with the same generator state and test every centroid
    rng = np.random.Generator(np.random.PCG64(4))
    centers, radii, vol = [], [], 0.0
    while vol < 0.2 * 4.0:
        r = rng.uniform(0.12, 0.3)
        c = rng.uniform([r, r, r], [4.0 - r, 1.0 - r, 1.0 - r])
        if centers and np.any(np.linalg.norm(np.asarray(centers) - c, axis=1) < np.asarray(radii) + r):
            continue
        centers.append(c)
        radii.append(r)
        vol += 4.0 / 3.0 * np.pi * r ** 3
    cent = p.coords[p.conn].mean(axis=1)
    d2 = ((cent[:, None, :] - np.asarray(centers)[None]) ** 2).sum(-1)
    inside = np.any(d2 <= np.asarray(radii)[None] ** 2, axis=1)
    assert np.array_equal(p.mat_id.astype(bool), inside)


def test_batched_blocks_ranges():
    probs = meshgen.batched_blocks(16, seed=11)
    for q in probs:
        nz, nx, ny = q.meta["nx"], q.meta["ny"], q.meta["nz"]
        assert 16 <= nz <= 64 and 4 <= nx <= 16 and 4 <= ny <= 16
        assert 0.1 <= q.mats[0, 0] <= 10.0 and 0.30 <= q.meta["nu"] <= 0.49


def _rsa_plain(seed, vol_frac, r_range, lx=4.0, ly=1.0, lz=1.0):
    """List-based random sequential addition: the generator's placement, restated plainly."""
    rng = np.random.Generator(np.random.PCG64(seed))
    centers, radii, vol = [], [], 0.0
    while vol < vol_frac * lx * ly * lz:
        r = rng.uniform(*r_range)
        c = rng.uniform([r, r, r], [lx - r, ly - r, lz - r])
        if centers and np.any(np.linalg.norm(np.asarray(centers) - c, axis=1) < np.asarray(radii) + r):
            continue
        centers.append(c)
        radii.append(r)
        vol += 4.0 / 3.0 * np.pi * r ** 3
    return len(radii), vol


def test_two_phase_placement_is_the_seeded_rsa():
    # the two-phase workload's layout (seed 23) and a training layout (seed 1000)
    for seed in (23, 1000):
        p = meshgen.two_phase_inclusions(32, 8, 8, seed=seed)
        n, vol = _rsa_plain(seed, 0.2, (0.03, 0.08))
        assert p.meta["n_spheres"] == n
        assert abs(p.meta["vol_frac"] - vol / 4.0) < 1e-15

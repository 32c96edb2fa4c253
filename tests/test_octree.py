"""Host octree / node-table properties (the mesh the GPU path takes as input)."""
import numpy as np
import pytest

from cudanextgenpb_b200 import configs

ROOT = 1 << 19


def morton(p):
    k = 0
    for b in range(20):
        for a in range(3):
            k |= ((int(p[a]) >> b) & 1) << (3 * b + a)
    return k


@pytest.fixture(scope="module")
def born_mesh():
    prob = configs.make_born_problem(5, 6).build()
    return prob, prob.mesh(), prob.info()


def test_born_mesh_counts(born_mesh):
    prob, m, info = born_mesh
    assert info["mesh_shape"] == 2 and info["unilevel"] == 5 and info["maxlevel"] == 6
    lv = m["oct_level"]
    assert set(np.unique(lv)) <= {5, 6}
    assert (lv == 6).sum() > 0
    # volume of the octants covers the root exactly
    size = (1 << (19 - lv.astype(np.int64))).astype(np.float64)
    assert np.isclose((size ** 3).sum(), float(ROOT) ** 3)


def test_octants_morton_sorted_and_aligned(born_mesh):
    _, m, _ = born_mesh
    xyz, lv = m["oct_xyz"], m["oct_level"].astype(np.int64)
    size = 1 << (19 - lv)
    assert np.all(xyz % size[:, None] == 0)
    keys = [morton(p) for p in xyz[:2000]]
    assert all(a < b for a, b in zip(keys, keys[1:]))


def test_balance_2to1(born_mesh):
    """Octants sharing a face, edge or corner differ by at most one level."""
    _, m, _ = born_mesh
    xyz, lv = m["oct_xyz"].astype(np.int64), m["oct_level"].astype(np.int64)
    size = 1 << (19 - lv)
    lo, hi = xyz, xyz + size[:, None]
    fine = np.where(lv == lv.max())[0][:400]
    coarse = np.where(lv == lv.min())[0]
    for i in fine:
        touch = np.all((lo[coarse] <= hi[i]) & (hi[coarse] >= lo[i]), axis=1)
        assert np.all(lv[i] - lv[coarse[touch]] <= 1)


def test_node_table(born_mesh):
    _, m, _ = born_mesh
    n, nh = m["n_nodes"], m["n_hang"]
    nodes, on = m["node_xyz"], m["oct_nodes"]
    # independent nodes in strictly increasing Morton order of their coordinates
    keys = [morton(p) for p in nodes[:3000]]
    assert all(a < b for a, b in zip(keys, keys[1:]))
    # each octant corner maps to a node at that corner's coordinates
    xyz, lv = m["oct_xyz"].astype(np.int64), m["oct_level"].astype(np.int64)
    size = 1 << (19 - lv)
    for o in range(0, len(xyz), 97):
        for c in range(8):
            p = xyz[o] + size[o] * np.array([c & 1, (c >> 1) & 1, (c >> 2) & 1])
            nd = on[o, c]
            if nd < n:
                assert np.array_equal(nodes[nd], p)
    # hanging parents are independent, and the hanging point is their midpoint
    par, np_ = m["hang_par"], m["hang_np"]
    assert set(np.unique(np_)) <= {2, 4}
    assert nh > 0
    for h in range(nh):
        k = np_[h]
        assert np.all(par[h, :k] >= 0) and np.all(par[h, :k] < n)
    # midpoint check through the octants that use the hanging node
    for o in range(len(xyz)):
        for c in range(8):
            nd = on[o, c]
            if nd >= n:
                h = nd - n
                p = xyz[o] + size[o] * np.array([c & 1, (c >> 1) & 1, (c >> 2) & 1])
                mid = nodes[par[h, :np_[h]]].mean(axis=0)
                assert np.array_equal(mid, p)


def test_ray_tables_sorted(born_mesh):
    prob, _, info = born_mesh
    for a in range(3):
        r = prob.rays(a)
        assert len(r["keys"]) == info["n_rays"][a] > 0
        assert np.all(np.diff(r["keys"].astype(np.float64)) > 0)
        cnt = np.diff(r["ptr"])
        assert np.all(cnt > 0) and np.all(cnt % 2 == 0)  # closed surface: entries pair with exits
        # normals are unit vectors
        assert np.allclose(np.linalg.norm(r["normals"], axis=1), 1.0)


def test_pqr_reader_dummy_atoms(tmp_path):
    from cudanextgenpb_b200 import Problem
    p = tmp_path / "one.pqr"
    p.write_text("ATOM      1  X    X     1      0.000   0.000    0.000  1.000 2.000\n")
    prob = Problem(configs.born_options())
    prob.read_pqr(str(p))
    pos, q, r = prob.atoms()
    # one atom plus 6 neutral zero-radius dummies at +-0.001 A (src/pb_class.cpp:1111-1149)
    assert len(q) == 7 and q[0] == 1.0 and np.all(q[1:] == 0) and np.all(r[1:] == 0)
    assert np.allclose(np.abs(pos[1:]).sum(axis=1), 0.001)


def test_pqr_reader_chain_and_radius(tmp_path):
    from cudanextgenpb_b200 import Problem
    p = tmp_path / "four.pqr"
    p.write_text("ATOM 1 N THR A 1 1.0 2.0 3.0 0.5 1.5\n"
                 "ATOM 2 CA THR 1 2.0 2.0 3.0 -0.5 0.0\n"
                 "ATOM 3 C THR 1 3.0 2.0 3.0 0.25 1.7\n"
                 "ATOM 4 O THR 1 4.0 2.0 3.0 -0.25 1.6\n"
                 "END\n")
    prob = Problem(configs.born_options())
    prob.read_pqr(str(p))
    pos, q, r = prob.atoms()
    assert len(q) == 4
    assert np.allclose(pos[0], [1, 2, 3]) and r[1] == 1.0  # radius < 1e-5 -> 1.0

"""VTU output of a node field (the reference's VTKWriter layout,
src/vtk_class.cpp:20-429), checked on the CPU against the host mesh: the
points are the independent nodes in id order, then one point per hanging
corner carrying its parents' mean; one voxel (type 11) per octant."""
import numpy as np

from cudanextgenpb_b200 import configs
from vtu_reader import read_vtu


def test_vtu_layout_matches_mesh(tmp_path):
    prob = configs.make_globular_problem(60, 7.0, -3.0, seed=60, levels=1).build()
    m = prob.mesh()
    n = m["n_nodes"]
    values = np.sin(np.arange(n) * 0.37)
    path = prob.write_vtu(str(tmp_path / "potential_map"), "phi", values)
    v = read_vtu(path)
    on = m["oct_nodes"]
    hang = on >= n
    n_pts = n + int(hang.sum())
    assert v["n_points"] == n_pts and v["n_cells"] == m["n_oct"]
    arr = v["arrays"]
    assert set(arr) == {"Array", "connectivity", "offsets", "types", "phi"}
    pts, conn, phi = arr["Array"], arr["connectivity"].reshape(-1, 8), arr["phi"]
    assert pts.shape == (n_pts, 3) and len(phi) == n_pts
    np.testing.assert_array_equal(arr["offsets"], 8 * np.arange(1, m["n_oct"] + 1))
    assert np.all(arr["types"] == 11)
    lo, ext = m["lo"], m["hi"] - m["lo"]
    # independent nodes: id order, coordinates and values
    np.testing.assert_array_equal(pts[:n], lo + ext * (m["node_xyz"] * 2.0 ** -19))
    np.testing.assert_array_equal(phi[:n], values)
    np.testing.assert_array_equal(conn[~hang], on[~hang])
    # hanging corners: one new point each, in octant-corner order
    np.testing.assert_array_equal(conn[hang], np.arange(n, n_pts))
    o_idx, c_idx = np.nonzero(hang)
    size = (1 << (19 - m["oct_level"][o_idx].astype(np.int64)))[:, None]
    bits = np.stack([(c_idx >> a) & 1 for a in range(3)], axis=1)
    corner = m["oct_xyz"][o_idx] + bits * size
    np.testing.assert_array_equal(pts[n:], lo + ext * (corner * 2.0 ** -19))
    h = on[hang] - n
    par, npar = m["hang_par"][h], m["hang_np"][h]
    mean = np.array([values[p[:k]].sum() / k for p, k in zip(par, npar)])
    np.testing.assert_allclose(phi[n:], mean, rtol=1e-15, atol=0)

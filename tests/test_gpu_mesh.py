"""Mesh construction on the GPU (pbgpu_build_mesh): surface refinement, nodes
with hanging nodes and ray tables built on the device from the initial
octree.  The host build of the same problem is the reference: identical
sizes, identical markers, fractions, matrix, right-hand side, potential and
energies."""
import numpy as np
import pytest

from cudanextgenpb_b200 import GpuPath, configs, solver_opts

pytestmark = pytest.mark.gpu

CASES = {
    "born": lambda: configs.make_born_problem(5, 6),
    "born_uniform": lambda: configs.make_born_problem(5, 5),
    "mol60": lambda: configs.make_globular_problem(60, 7.0, -3.0, seed=60, levels=1),
    "mol150": lambda: configs.make_globular_problem(150, 9.0, 2.0, seed=150, levels=2),
    "mol300": lambda: configs.make_globular_problem(300, 11.0, -3.0, seed=300, levels=2),
}


@pytest.mark.parametrize("name", sorted(CASES))
def test_gpu_mesh_equals_host_mesh(name):
    host = CASES[name]().build()
    info = host.info()
    g_host = GpuPath().load(host)
    g_dev = CASES[name]().build_on_gpu(GpuPath())
    assert (g_dev.n_oct, g_dev.n, g_dev.n_hang) == (info["n_oct"], info["n_nodes"], info["n_hang"])
    assert g_dev.n_rays == list(info["n_rays"])
    # the arrays themselves, read back from both contexts
    hm = host.mesh()
    for g in (g_host, g_dev):
        d = g.mesh_arrays()
        for k in ("oct_xyz", "oct_level", "oct_nodes", "node_xyz", "hang_np", "hang_par"):
            assert np.array_equal(d[k], hm[k]), k
        np.testing.assert_array_equal(d["lo"], hm["lo"])
    for g in (g_host, g_dev):
        g.create_markers()
        g.create_density_map()
        g.assemble()
    mh, bh = g_host.markers()
    md, bd = g_dev.markers()
    assert np.array_equal(mh, md) and np.array_equal(bh, bd)
    assert np.array_equal(g_host.fractions(len(bh)), g_dev.fractions(len(bd)))
    for a, b in zip(g_host.system(), g_dev.system()):
        assert np.array_equal(a, b)
    opts = solver_opts("cg", tol=1e-10)
    g_host.solve(opts)
    g_dev.solve(opts)
    assert np.array_equal(g_host.phi(), g_dev.phi())
    eh, ed = g_host.energy(), g_dev.energy()
    for k in ("energy_pol", "energy_react", "energy_coul", "charge_flux"):
        assert eh[k] == ed[k], k
    g_host.close()
    g_dev.close()


@pytest.mark.parametrize("name", ["born", "mol60", "mol150"])
def test_initial_octree_on_gpu_equals_host_initial_octree(name):
    """init_tmesh* on the GPU (n_oct = 0: uniform level, then box refinement
    with 2:1 balance) and on the host give the same refined mesh."""
    p_host, p_dev = CASES[name](), CASES[name]()
    b_host, b_dev = p_host.mesh_build(on_gpu=False), p_dev.mesh_build(on_gpu=True)
    assert b_host.n_oct > 0 and b_dev.n_oct == 0
    g_host, g_dev = GpuPath().build_mesh(b_host), GpuPath().build_mesh(b_dev)
    assert (g_host.n_oct, g_host.n, g_host.n_hang) == (g_dev.n_oct, g_dev.n, g_dev.n_hang)
    assert g_host.n_rays == g_dev.n_rays
    dh, dd = g_host.mesh_arrays(), g_dev.mesh_arrays()
    for k in ("oct_xyz", "oct_level", "oct_nodes", "node_xyz", "hang_np", "hang_par", "lo", "extent"):
        assert np.array_equal(dh[k], dd[k]), k
    g_host.close()
    g_dev.close()

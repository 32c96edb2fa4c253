"""Parity of the sm_100a path with the CPU oracle, stage by stage, on the same
seeded inputs.  Integer / index results must be identical; values that the GPU
computes with the oracle's own expressions (markers, fractions, density) must be
bit-identical; assembled values within 1e-12 relative; potentials within 1e-6
relative L2 of a tight solve; energies within 1e-6 relative (1e-10 when both
sides use the same potential)."""
import numpy as np
import pytest

from cudanextgenpb_b200 import GpuPath, configs, solver_opts
from cudanextgenpb_b200 import _native as N
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu

CASES = {
    "born": lambda: configs.make_born_problem(5, 6),
    "mol60": lambda: configs.make_globular_problem(60, 7.0, -3.0, seed=60, levels=1),
    "mol150": lambda: configs.make_globular_problem(150, 9.0, 2.0, seed=150, levels=2),
}


def _prep(name):
    prob = CASES[name]().build()
    o = Oracle(prob)
    g = GpuPath().load(prob)
    return prob, o, g


@pytest.fixture(scope="module", params=sorted(CASES))
def case(request):
    prob, o, g = _prep(request.param)
    om, ob = o.markers()
    o.density()
    osys = o.assemble()
    g.create_markers()
    g.create_density_map()
    g.assemble()
    yield request.param, prob, o, g, (om, ob), osys
    g.close()
    o.close()


def test_markers_exact(case):
    name, prob, o, g, (om, ob), _ = case
    gm, gb = g.markers()
    assert np.array_equal(gm, om)
    assert np.array_equal(gb, ob)
    ge, gr = g.node_coeffs()
    oe, orr = o.node_coeffs()
    assert np.array_equal(ge, oe) and np.array_equal(gr, orr)


def test_fractions_exact(case):
    name, prob, o, g, (om, ob), _ = case
    assert np.array_equal(g.fractions(len(ob)), o.fractions(len(ob)))


def test_density_exact(case):
    name, prob, o, g, _, _ = case
    grho, gvp = g.density()
    orho, ovp = o.density()
    assert np.array_equal(gvp, ovp)
    assert np.array_equal(grho, orho)
    assert abs((grho * gvp).sum() / (4 * np.pi) - prob.info()["net_charge"]) < 1e-9


def test_system_pattern_exact_values_close(case):
    name, prob, o, g, _, (orp, ocol, oval, orhs) = case
    grp, gcol, gval, grhs = g.system()
    assert np.array_equal(grp, orp)
    assert np.array_equal(gcol, ocol)
    scale = np.abs(oval).max()
    assert np.max(np.abs(gval - oval)) <= 1e-12 * scale
    assert np.max(np.abs(grhs - orhs)) <= 1e-12 * max(np.abs(orhs).max(), 1e-300)


@pytest.mark.parametrize("method", ["cg", "bicgstab"])
def test_solve_and_energy(case, method):
    name, prob, o, g, _, _ = case
    st = g.solve(solver_opts(method, tol=1e-10, max_iter=20000))
    assert st.status == 0 and st.rel_residual < 2e-10
    gphi = g.phi()
    ophi, it, rel = o.solve("cg", 1e-12)
    err = np.linalg.norm(gphi - ophi) / np.linalg.norm(ophi)
    assert err < 1e-6, err
    fast = name == "uniform"
    ge = g.energy(fast)
    oe = o.energy(fast)
    for k in ("energy_pol", "energy_react", "energy_coul", "sum"):
        assert ge[k] == pytest.approx(oe[k], rel=1e-6, abs=1e-9), k
    # same potential on both sides: the energy kernels agree much more tightly
    o.set_phi(gphi)
    oe2 = o.energy(fast)
    for k in ("energy_pol", "energy_react", "energy_coul", "charge_flux"):
        assert ge[k] == pytest.approx(oe2[k], rel=1e-10, abs=1e-12), k
    gpa = g.phi_on_atoms()
    opa = o.phi_on_atoms()
    ok = ~np.isnan(opa)
    assert np.array_equal(np.isnan(gpa), np.isnan(opa))
    assert np.allclose(gpa[ok], opa[ok], rtol=1e-12, atol=1e-14)


def test_mixed_precision(case):
    name, prob, o, g, _, _ = case
    st = g.solve(solver_opts("cg", tol=1e-10, precision="mixed", inner_tol=1e-4))
    assert st.status == 0 and st.rel_residual < 1e-10 and st.outer >= 2
    gphi = g.phi()
    ophi, it, rel = o.solve("cg", 1e-12)
    assert np.linalg.norm(gphi - ophi) / np.linalg.norm(ophi) < 1e-6
    ge, oe = g.energy(), o.energy()
    assert ge["sum"] == pytest.approx(oe["sum"], rel=1e-6)


def test_born_gpu_vs_analytic():
    prob = configs.make_born_problem(5, 6).build()
    g = GpuPath().load(prob)
    e, st = g.run(solver_opts("bicgstab", tol=1e-8))
    assert st.status == 0
    ref = configs.born_energy()
    assert abs(e["sum"] - ref) / abs(ref) < 5e-4
    assert abs(e["charge_flux"] - 1.0) < 1e-5


def test_uniform_mesh_energy_fast():
    prob = configs.make_born_problem(5, 5).build()
    o = Oracle(prob)
    oe, ophi, _, _ = o.run("cg", 1e-12, fast=True)
    g = GpuPath().load(prob)
    ge, st = g.run(solver_opts("cg", tol=1e-11), fast=True)
    for k in ("energy_pol", "energy_react"):
        assert ge[k] == pytest.approx(oe[k], rel=1e-7)


@pytest.mark.parametrize("chunk,sigma,group", [(32, 1, 1), (64, 64, 2), (32, 512, 4), (128, 1024, 1),
                                               (32, 2048, 2), (32, 32, 4)])
def test_sell_layouts_agree(chunk, sigma, group):
    prob = CASES["mol60"]().build()
    o = Oracle(prob)
    o.markers()
    o.density()
    orp, ocol, oval, orhs = o.assemble()
    g = GpuPath().load(prob)
    g.create_markers()
    g.create_density_map()
    g.assemble(chunk, sigma, group)
    grp, gcol, gval, grhs = g.system()
    assert np.array_equal(grp, orp) and np.array_equal(gcol, ocol)
    assert np.max(np.abs(gval - oval)) <= 1e-12 * np.abs(oval).max()
    st = g.solve(solver_opts("cg", tol=1e-10))
    ophi, _, _ = o.solve("cg", 1e-12)
    assert np.linalg.norm(g.phi() - ophi) / np.linalg.norm(ophi) < 1e-6


@pytest.mark.parametrize("bc", [0, 1, 2])
def test_boundary_condition_types(bc):
    prob = configs.make_born_problem(4, 5, bc_type=bc).build()
    o = Oracle(prob)
    o.markers()
    o.density()
    orp, ocol, oval, orhs = o.assemble()
    g = GpuPath().load(prob)
    g.create_markers()
    g.create_density_map()
    g.assemble()
    grp, gcol, gval, grhs = g.system()
    assert np.array_equal(grp, orp) and np.array_equal(gcol, ocol)
    assert np.max(np.abs(grhs - orhs)) <= 1e-12 * np.abs(orhs).max()


def test_stern_layer():
    prob = configs.make_globular_problem(60, 7.0, -3.0, seed=61, levels=1)
    prob.set_option("surface/stern_layer_surf", 1)
    prob.set_option("surface/stern_layer_thickness", 2.0)
    prob.build()
    o = Oracle(prob)
    om, ob = o.markers()
    o.density()
    orp, ocol, oval, orhs = o.assemble()
    g = GpuPath().load(prob)
    g.create_markers()
    g.create_density_map()
    g.assemble()
    gm, gb = g.markers()
    assert np.array_equal(gm, om)
    grp, gcol, gval, grhs = g.system()
    assert np.array_equal(grp, orp) and np.array_equal(gcol, ocol)
    assert np.max(np.abs(gval - oval)) <= 1e-12 * np.abs(oval).max()


def test_call_order_and_iteration_cap():
    prob = configs.make_born_problem(4, 5).build()
    g = GpuPath().load(prob)
    lib = N.load_gpu()
    assert lib.pbgpu_solve(g._ctx, None, None) == N.PBGPU_ERR_STATE
    assert lib.pbgpu_assemble(g._ctx, None) == N.PBGPU_ERR_STATE
    g.create_markers()
    g.create_density_map()
    g.assemble()
    st = g.solve(solver_opts("cg", tol=1e-14, max_iter=5), allow_not_converged=True)
    assert st.status == N.PBGPU_NOT_CONVERGED and st.iterations == 5
    # the context stays usable
    st = g.solve(solver_opts("cg", tol=1e-8))
    assert st.status == 0


def test_repeated_full_path_on_one_context():
    """The whole path run three times on one context gives the same results
    (the pattern of a serving loop and of the benchmark's steps).  Everything up
    to the potential is bit-reproducible; the energy adds per-crossing
    coefficients with atomics, so it agrees to rounding."""
    prob = CASES["mol60"]().build()
    g = GpuPath().load(prob)
    opts = solver_opts("cg", tol=1e-8, max_iter=50000)
    out = []
    for _ in range(3):
        g.create_markers()
        g.create_density_map()
        g.assemble()
        st = g.solve(opts)
        pa = g.phi_on_atoms()
        e = g.energy(False)
        out.append((st.iterations, e["sum"], pa.copy()))
    for it, es, pa in out[1:]:
        assert it == out[0][0] and np.array_equal(pa, out[0][2])
        assert es == pytest.approx(out[0][1], rel=1e-13)


def test_host_driver_path_matches():
    """pbhost_run_gpu (the C++ pb_class mirror's driver order) gives the same energy."""
    prob = configs.make_born_problem(5, 6).build()
    e_host, st = prob.run_gpu()
    g = GpuPath().load(prob)
    opts = prob.solver_opts()
    e, st2 = g.run(opts)
    assert e_host["sum"] == pytest.approx(e["sum"], rel=1e-9)

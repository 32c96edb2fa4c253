"""Edge cases of the path, on the GPU against the oracle.

* A molecule without charge: the right-hand side is zero (Coulomb boundary
  values of zero charges), so every solver returns x = 0 at once, as LIS does
  for a zero right-hand side, and every energy, potential at an atom and
  pot_field column is 0.
* An atom outside the mesh: it adds no density, its potential is NaN (the
  reference's atom search finds no octant for it, src/pb_class.cpp:3633-3729),
  and the energies still count its charge, as the reference's pair sums do."""
import numpy as np
import pytest

from cudanextgenpb_b200 import Batch, GpuPath, configs, solver_opts
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu


def _mol60(zero_charge=False):
    prob = configs.make_globular_problem(60, 7.0, -3.0, seed=60, levels=1)
    if zero_charge:
        pos, q, r = configs.synthetic_molecule(60, 7.0, -3.0, 60)
        prob.set_atoms(pos, np.zeros_like(q), r)
    return prob.build()


def _setup(g):
    g.create_markers()
    g.create_density_map()
    g.assemble()


@pytest.mark.parametrize("method,precision", [("cg", "fp64"), ("bicgstab", "fp64"), ("cgs", "fp64"),
                                              ("cg", "mixed"), ("bicgstab", "mixed")])
def test_uncharged_molecule_solves_to_zero(method, precision):
    prob = _mol60(zero_charge=True)
    g = GpuPath().load(prob)
    _setup(g)
    st = g.solve(solver_opts(method, tol=1e-10, precision=precision))
    assert st.status == 0 and st.iterations == 0
    assert np.all(g.phi() == 0.0)
    e = g.energy()
    for k in ("energy_pol", "energy_react", "energy_coul", "charge_flux", "sum"):
        assert e[k] == 0.0, k
    assert np.all(g.phi_on_atoms() == 0.0)
    rows, pe = g.pot_field(2, 2)
    assert np.all(rows == 0.0) and pe["energy_pol"] == 0.0 and pe["energy_react"] == 0.0
    g.close()
    o = Oracle(prob)
    oe, ophi, _, _ = o.run("cg", 1e-12)
    assert np.all(ophi == 0.0) and oe["sum"] == 0.0
    o.close()


def test_uncharged_molecule_in_a_batch():
    g0 = GpuPath().load(_mol60(zero_charge=True))
    g1 = GpuPath().load(_mol60())
    for g in (g0, g1):
        _setup(g)
    ref = GpuPath().load(_mol60())
    _setup(ref)
    ref.solve(solver_opts("cg", tol=1e-10))
    b = Batch()
    b.add(g0)
    b.add(g1)
    stats = b.solve(solver_opts("cg", tol=1e-10))
    assert all(s.status == 0 for s in stats.values())
    assert np.all(g0.phi() == 0.0)
    assert g1.energy()["sum"] == pytest.approx(ref.energy()["sum"], rel=1e-6)
    b.close()
    for g in (g0, g1, ref):
        g.close()


def test_atom_outside_the_mesh():
    prob = _mol60()
    pos, q, _ = prob.atoms()
    pos2 = np.vstack([pos, [[500.0, 0.0, 0.0]]])
    q2 = np.append(q, 1.0)
    g = GpuPath().load(prob)
    g.set_atoms(pos2, q2)
    _setup(g)
    o = Oracle(prob, atoms=(pos2, q2))
    o.markers()
    orho, ovp = o.density()
    grho, gvp = g.density()
    assert np.array_equal(grho, orho) and np.array_equal(gvp, ovp)
    # the outside atom adds nothing: the density is that of the molecule alone
    g_in = GpuPath().load(prob)
    _setup(g_in)
    assert np.array_equal(g_in.density()[0], grho)
    o.assemble()
    st = g.solve(solver_opts("cg", tol=1e-11))
    assert st.status == 0
    ophi, _, _ = o.solve("cg", 1e-12)
    assert np.linalg.norm(g.phi() - ophi) / np.linalg.norm(ophi) < 1e-6
    gpa, opa = g.phi_on_atoms(), o.phi_on_atoms()
    assert np.isnan(gpa[-1]) and np.isnan(opa[-1])
    assert np.allclose(gpa[:-1], opa[:-1], rtol=1e-6)
    o.set_phi(g.phi())
    ge, oe = g.energy(), o.energy()
    for k in ("energy_pol", "energy_react", "energy_coul"):
        assert ge[k] == pytest.approx(oe[k], rel=1e-10, abs=1e-12), k
    rows, pe = g.pot_field(2, 2)
    orows, ope = o.pot_field(2, 2)
    for k in ("energy_pol", "energy_react", "energy_coul"):
        assert pe[k] == pytest.approx(ope[k], rel=1e-10, abs=1e-12), k
    scale = np.abs(orows).max(axis=0)
    assert np.all(np.abs(rows - orows) <= 1e-9 * np.maximum(scale, 1e-300))
    o.close()
    g.close()
    g_in.close()

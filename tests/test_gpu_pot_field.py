"""pot_field / pot_field_fast on the GPU against the CPU oracle's restatement
of the reference's element loops (src/pb_class.cpp:3732-5060).

Both sides use the same potential, so the only differences are the order of
the sums (the GPU merges the elements on a crossing and sums per atom) and the
last bits of the surface point coordinates.  Per-atom columns must agree to
1e-9 of the size of their summands: a potential column to 1e-9 of its
largest magnitude, a field column to 1e-9 of the largest of its part's field
and potential (per angstrom) -- a field that cancels to almost nothing, as
the reaction field inside the Born sphere does, keeps only rounding noise of
the terms.  Energies agree to 1e-10 relative, and the set of written columns
is identical for every option pair."""
import numpy as np
import pytest

from cudanextgenpb_b200 import GpuPath, Problem, configs, solver_opts
from cudanextgenpb_b200 import _native as N
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu

SALT_FREE = configs.born_options(5, 6).replace("ionic_strength = 0.145", "ionic_strength = 0")

CASES = {
    "born": (lambda: configs.make_born_problem(5, 6), False),
    "born_salt_free": (lambda: _born_salt_free(), False),
    "born_uniform": (lambda: configs.make_born_problem(5, 5), True),
    "mol60": (lambda: configs.make_globular_problem(60, 7.0, -3.0, seed=60, levels=1), False),
    "mol150": (lambda: configs.make_globular_problem(150, 9.0, 2.0, seed=150, levels=2), False),
}

OPTION_PAIRS = [(pt, ft) for pt in range(3) for ft in range(3)]


def _born_salt_free():
    p = Problem(SALT_FREE)
    p.set_atoms(*configs.BORN_ATOM)
    return p


@pytest.fixture(scope="module", params=sorted(CASES))
def solved(request):
    make, fast = CASES[request.param]
    prob = make().build()
    g = GpuPath().load(prob)
    g.create_markers()
    g.create_density_map()
    g.assemble()
    st = g.solve(solver_opts("cg", tol=1e-11, max_iter=20000))
    assert st.status == 0
    o = Oracle(prob)
    o.markers()
    o.density()
    o.assemble()
    o.set_phi(g.phi())
    yield request.param, fast, prob, g, o
    g.close()
    o.close()


PART = {"c": (0, 3, 4, 5), "p": (1, 6, 7, 8), "i": (2, 9, 10, 11)}


def _close_columns(gr, orows, columns):
    for k, name in enumerate(N.POT_FIELD_COLUMNS):
        if not (columns >> k) & 1:
            assert np.all(gr[:, k] == 0.0) and np.all(orows[:, k] == 0.0), name
            continue
        scale = np.abs(orows[:, k]).max()
        if name.startswith("E"):
            cols = list(PART[name[-1]])
            scale = max(scale, np.abs(orows[:, cols]).max())
        scale = max(scale, 1e-300)
        err = np.abs(gr[:, k] - orows[:, k]).max()
        assert err <= 1e-9 * scale, (name, err, scale)


@pytest.mark.parametrize("pt,ft", OPTION_PAIRS)
def test_pot_field_matches_oracle(solved, pt, ft):
    name, fast, prob, g, o = solved
    gr, ge = g.pot_field(pt, ft, fast=fast)
    orows, oe = o.pot_field(pt, ft, fast=fast)
    assert ge["columns"] == oe["columns"]
    _close_columns(gr, orows, oe["columns"])
    for k in ("energy_pol", "energy_react", "energy_coul", "charge_flux"):
        assert ge[k] == pytest.approx(oe[k], rel=1e-10, abs=1e-12), k


def test_pot_field_energies_equal_energy(solved):
    """The per-atom sums carry the energy routine's polarisation (and, with
    salt, ionic) energy and flux charge; the Coulomb energy is half the sum of
    q phi_c, and equals the energy routine's whenever that one is computed."""
    name, fast, prob, g, o = solved
    salt = name != "born_salt_free"
    rows, pe = g.pot_field(*((2, 2) if salt else (1, 1)), fast=fast)
    e = g.energy(fast)
    for k in ("energy_pol", "energy_react", "charge_flux") if salt else ("energy_pol", "charge_flux"):
        assert pe[k] == pytest.approx(e[k], rel=1e-10, abs=1e-12), k
    _, q, _ = prob.atoms()
    assert pe["energy_coul"] == pytest.approx(0.5 * (q * rows[:, 0]).sum(), rel=1e-12, abs=1e-12)
    if e["energy_coul"] != 0.0:
        assert pe["energy_coul"] == pytest.approx(e["energy_coul"], rel=1e-10)


def test_pot_field_rejects_bad_options():
    g = GpuPath().load(configs.make_born_problem(4, 5).build())
    with pytest.raises(Exception):
        g.pot_field(0, 0)  # before a solve
    g.create_markers()
    g.create_density_map()
    g.assemble()
    g.solve(solver_opts("cg", tol=1e-8))
    for pt, ft in ((3, 0), (0, -1)):
        with pytest.raises(Exception):
            g.pot_field(pt, ft)
    g.close()


def test_host_driver_writes_pot_field(tmp_path, monkeypatch):
    """With calc_potential_terms / calc_field_terms set, the host mirror's
    driver runs pot_field (refined mesh) instead of energy and writes
    pot_field.dat in the reference's layout: a heading naming the written
    columns, then one row per atom, every value in %8g."""
    text = configs.born_options(5, 6).replace(
        "calc_coulombic = 1", "calc_coulombic = 1\ncalc_potential_terms = 2\ncalc_field_terms = 1")
    prob = Problem(text)
    prob.set_atoms(*configs.BORN_ATOM)
    prob.build()
    monkeypatch.chdir(tmp_path)
    e, st = prob.run_gpu()
    lines = (tmp_path / "pot_field.dat").read_text().splitlines()
    assert lines[0] == ("# index    x    y    z    phi_c    phi_p    phi_i    Ex_c    Ey_c    Ez_c   "
                        "Ex_p    Ey_p    Ez_p")
    pos, q, _ = prob.atoms()
    assert len(lines) == 1 + len(q)
    g = GpuPath().load(prob)
    g.create_markers()
    g.create_density_map()
    g.assemble()
    g.solve(prob.solver_opts())
    rows, pe = g.pot_field(2, 1)
    cols = [k for k in range(len(N.POT_FIELD_COLUMNS)) if (pe["columns"] >> k) & 1]
    assert len(cols) == 9
    # 6 significant digits; sums that cancel to rounding noise (the reaction
    # field at the ion) vary in their last bits between runs
    colmax = np.abs(rows[:, cols]).max(axis=0)
    for i, line in enumerate(lines[1:]):
        f = line.split()
        assert int(f[0]) == i + 1
        assert np.allclose([float(x) for x in f[1:4]], pos[i], rtol=1e-5, atol=1e-9)
        vals = np.array([float(x) for x in f[4:]])
        assert len(vals) == len(cols)
        assert np.all(np.abs(vals - rows[i, cols]) <= 6e-6 * np.abs(rows[i, cols]) + 1e-9 * colmax)
    assert e["energy_pol"] == pytest.approx(pe["energy_pol"], rel=1e-6)
    assert e["energy_react"] == pytest.approx(pe["energy_react"], rel=1e-6)
    g.close()


def test_host_driver_writes_vtu_maps(tmp_path, monkeypatch):
    """potential_map / eps_map with map_type = vtu: the driver writes
    potential_map_0000.vtu (phi), eps_map_0000.vtu (epsilon at the nodes) and
    their total_*.pvtu, from the context's own potential; with the mesh built
    on the GPU the same files come from the context's mesh."""
    from vtu_reader import read_vtu
    text = configs.born_options(5, 6).replace(
        "calc_coulombic = 1", "calc_coulombic = 1\npotential_map = 1\neps_map = 1\nmap_type = vtu")
    prob = Problem(text)
    prob.set_atoms(*configs.BORN_ATOM)
    prob.build()
    monkeypatch.chdir(tmp_path)
    prob.run_gpu()
    g = GpuPath().load(prob)
    g.create_markers()
    g.create_density_map()
    g.assemble()
    g.solve(prob.solver_opts())
    n = g.n
    phi = read_vtu("potential_map_0000.vtu")["arrays"]["phi"]
    eps = read_vtu("eps_map_0000.vtu")["arrays"]["eps"]
    np.testing.assert_array_equal(phi[:n], g.phi())
    np.testing.assert_array_equal(eps[:n], g.node_coeffs()[0])
    for base, field in (("potential_map", "phi"), ("eps_map", "eps")):
        t = (tmp_path / ("total_%s.pvtu" % base)).read_text()
        assert 'Name="%s"' % field in t and '<Piece Source="%s_0000.vtu"/>' % base in t
    g.close()
    # mesh built on the GPU: same file
    os_mesh = (tmp_path / "potential_map_0000.vtu").read_bytes()
    p2 = Problem(text)
    p2.set_atoms(*configs.BORN_ATOM)
    g2 = p2.build_on_gpu(GpuPath())
    g2.create_markers()
    g2.create_density_map()
    g2.assemble()
    g2.solve(prob.solver_opts())
    p2.write_vtu(str(tmp_path / "gpu_map"), "phi", g2.phi())
    assert (tmp_path / "gpu_map_0000.vtu").read_bytes() == os_mesh
    g2.close()

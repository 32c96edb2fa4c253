"""The CPU oracle against known answers: the analytic Born / Debye-Hueckel energy
of a charged sphere, Gauss's law, and self-consistency checks.  The reference
ships no tests or golden outputs of its own, so these are the pins."""
import json
import os

import numpy as np
import pytest
import scipy.sparse as sp
import scipy.sparse.linalg as spla

from cudanextgenpb_b200 import Problem, configs
from cudanextgenpb_b200._native import POT_FIELD_COLUMNS
from oracle_lib import Oracle

HERE = os.path.dirname(os.path.abspath(__file__))


@pytest.fixture(scope="module")
def born():
    prob = configs.make_born_problem(5, 6).build()
    o = Oracle(prob)
    o.markers()
    o.density()
    sysm = o.assemble()
    return prob, o, sysm


def test_born_constants_match_reference_values():
    eps_in, eps_out, k = configs.scaled_constants()
    # values of the reference's units at T = 298.15 K, I = 0.145 M
    assert abs(eps_in - 0.0035685016236776) < 1e-15
    assert abs(eps_out - 0.1427400649471059) < 1e-14
    assert abs(k - 0.1239941973227606) < 1e-14
    assert abs(configs.born_energy() - (-68.65400844521548)) < 1e-11
    assert abs(configs.born_energy(ionic=0.0) - (-68.30597984954667)) < 1e-11


def test_born_energy_vs_analytic(born):
    prob, o, _ = born
    phi, it, rel = o.solve("bicgstab", 1e-12)
    assert rel < 1e-11
    e = o.energy()
    ref = configs.born_energy()
    assert abs(e["sum"] - ref) / abs(ref) < 5e-4
    # the polarisation part is the salt-free Born energy
    assert abs(e["energy_pol"] - configs.born_energy(ionic=0.0)) / 68.3 < 1e-5
    # Gauss's law: the flux through the dielectric jump carries the enclosed charge
    assert abs(e["charge_flux"] - 1.0) < 1e-9
    assert e["net_charge"] == 1.0 and e["energy_coul"] == 0.0


def test_born_energy_converges():
    errs = []
    for u, m in ((4, 5), (5, 6), (6, 7)):
        prob = configs.make_born_problem(u, m).build()
        o = Oracle(prob)
        e, _, _, _ = o.run("cg", 1e-12)
        errs.append(abs(e["sum"] - configs.born_energy()))
    assert errs[2] < errs[1] < errs[0]
    assert errs[1] / errs[2] > 2.5  # second order in h


def test_matrix_symmetric_and_dirichlet_rows(born):
    prob, o, (rp, col, val, rhs) = born
    n = len(rp) - 1
    A = sp.csr_matrix((val, col, rp), shape=(n, n))
    assert abs(A - A.T).max() < 1e-12 * abs(A).max()
    m = prob.mesh()
    onb = np.any((m["node_xyz"] == 0) | (m["node_xyz"] == 1 << 19), axis=1)
    d = np.diff(rp)
    assert np.all(d[onb] == 1) and np.allclose(A.diagonal()[onb], 1.0)
    # positive diagonal; rows of a uniform region hold the 7-point stencil
    assert np.all(A.diagonal() > 0)
    assert np.median(d[~onb]) == 7
    # Dirichlet columns are eliminated from the other rows
    cols_of_interior = col[np.repeat(~onb, d)]
    assert not np.any(onb[cols_of_interior])


def test_krylov_vs_direct(born):
    prob, o, (rp, col, val, rhs) = born
    n = len(rp) - 1
    A = sp.csc_matrix(sp.csr_matrix((val, col, rp), shape=(n, n)))
    x = spla.spsolve(A, rhs)
    for meth in ("cg", "bicgstab"):
        phi, it, rel = o.solve(meth, 1e-12)
        assert np.linalg.norm(phi - x) / np.linalg.norm(x) < 1e-9


@pytest.mark.parametrize("case", ["born", "mol60"])
def test_two_oracle_assemblies_identical(case):
    """The triplet and the row-gather restatements of the assembly agree bit for
    bit (hanging-node meshes included)."""
    if case == "born":
        prob = configs.make_born_problem(5, 6).build()
    else:
        prob = configs.make_globular_problem(60, 7.0, -3.0, seed=60, levels=1).build()
    o = Oracle(prob)
    o.markers()
    o.density()
    a = o.assemble("triplets")
    b = o.assemble("rows")
    for x, y in zip(a, b):
        assert np.array_equal(x, y)


def test_energy_fast_equals_energy_on_uniform_mesh():
    # no surface refinement: a uniform mesh without hanging nodes
    prob = configs.make_born_problem(5, 5).build()
    assert prob.info()["n_hang"] == 0
    o = Oracle(prob)
    e, phi, it, rel = o.run("cg", 1e-12)
    ef = o.energy(fast=True)
    for k in ("energy_pol", "energy_react", "charge_flux"):
        assert ef[k] == pytest.approx(e[k], rel=1e-14, abs=1e-14)


def test_density_conserves_charge(born):
    prob, o, _ = born
    rho, vp = o.density()
    # the box integral of rho returns 4 pi q
    assert abs((rho * vp).sum() / (4 * np.pi) - 1.0) < 1e-12
    assert abs(vp.sum() - 16.0 ** 3) < 1e-9


def test_golden_born_fixture(born):
    """Regression pin of the oracle against its committed Born fixture
    (tests/golden/make_golden.py writes it)."""
    path = os.path.join(HERE, "golden", "born_u5_m6.json")
    g = json.load(open(path))
    prob, o, (rp, col, val, rhs) = born
    info = prob.info()
    assert [info["n_oct"], info["n_nodes"], info["n_hang"]] == g["mesh_counts"]
    marker, border = o.markers()
    assert len(border) == g["n_border"]
    assert int(rp[-1]) == g["nnz"]
    assert abs(val.sum() - g["sum_val"]) <= 1e-12 * abs(g["sum_val"])
    assert abs(rhs.sum() - g["sum_rhs"]) <= 1e-12 * abs(g["sum_rhs"])
    phi, it, rel = o.solve("cg", 1e-12)
    e = o.energy()
    for k in ("energy_pol", "energy_react", "charge_flux"):
        assert e[k] == pytest.approx(g["energy"][k], rel=1e-9)


@pytest.mark.parametrize("method", ["cg", "bicgstab"])
def test_preconditioners_same_solution(born, method):
    """-p none / jacobi / block Jacobi: the same solution, preconditioned runs
    need fewer iterations than the unpreconditioned one."""
    prob, o, _ = born
    ref, _, _ = o.solve("cg", 1e-12)
    its = {}
    for pc in ("none", "jacobi", "block_jacobi"):
        phi, it, rel = o.solve(method, 1e-10, precond=pc)
        assert rel <= 1e-10
        assert np.linalg.norm(phi - ref) / np.linalg.norm(ref) < 1e-8
        its[pc] = it
    assert its["jacobi"] < its["none"] and its["block_jacobi"] < its["none"]


def test_cgs_and_conv_cond(born):
    """CGS reaches the CG solution; conv_cond 2 (||r||_1 <= tol_w ||b||_1 +
    tol) stops on the 1-norm of the residual."""
    prob, o, (rp, col, val, rhs) = born
    ref, _, _ = o.solve("cg", 1e-12)
    for pc in ("jacobi", "block_jacobi"):
        phi, it, rel = o.solve("cgs", 1e-10, precond=pc)
        assert rel <= 1e-10 and np.linalg.norm(phi - ref) / np.linalg.norm(ref) < 1e-8
    n = len(rp) - 1
    A = sp.csr_matrix((val, col, rp), shape=(n, n))
    for tol in (1e-4, 1e-6):
        phi, it, rel = o.solve("cgs", tol, precond="block_jacobi", conv_cond=2, tol_w=0.0)
        assert np.abs(rhs - A @ phi).sum() <= 1.01 * tol
    # a looser rule stops earlier
    _, it4, _ = o.solve("cgs", 1e-4, precond="block_jacobi", conv_cond=2, tol_w=0.0)
    _, it6, _ = o.solve("cgs", 1e-6, precond="block_jacobi", conv_cond=2, tol_w=0.0)
    assert it4 < it6


def _born_pair(salt=True):
    text = configs.born_options(4, 5)
    if not salt:
        text = text.replace("ionic_strength = 0.145", "ionic_strength = 0")
    prob = Problem(text)
    prob.set_atoms(*configs.BORN_ATOM)
    o = Oracle(prob.build())
    o.markers()
    o.density()
    o.assemble()
    o.solve("cg", 1e-12)
    return o


def test_pot_field_column_sets():
    """pot_field writes the columns of the reference's print branches
    (src/pb_class.cpp:4281-4375), which depend on the options and on salt."""
    c = lambda *names: sum(1 << POT_FIELD_COLUMNS.index(n) for n in names)
    base = c("phi_c", "Ex_c", "Ey_c", "Ez_c")
    ep = c("Ex_p", "Ey_p", "Ez_p")
    ei = c("Ex_i", "Ey_i", "Ez_i")
    salt = {(0, 0): 0, (1, 0): base | c("phi_p"), (2, 0): base | c("phi_p", "phi_i"),
            (0, 1): base | c("phi_p") | ep, (1, 1): base | c("phi_p") | ep,
            (2, 1): base | c("phi_p", "phi_i") | ep,
            (0, 2): base | c("phi_p", "phi_i") | ep | ei, (1, 2): base | c("phi_p", "phi_i") | ep | ei,
            (2, 2): base | c("phi_p", "phi_i") | ep | ei}
    no_salt = {(0, 0): 0, (1, 0): base | c("phi_p"), (2, 0): base | c("phi_p"),
               (0, 1): base | c("phi_p") | ep, (1, 1): base | c("phi_p") | ep, (2, 1): 0,
               (0, 2): base | c("phi_p") | ep, (1, 2): base | c("phi_p") | ep, (2, 2): 0}
    for salty, table in ((True, salt), (False, no_salt)):
        o = _born_pair(salty)
        for (pt, ft), cols in table.items():
            rows, e = o.pot_field(pt, ft)
            assert e["columns"] == cols, (salty, pt, ft)
            for k in range(len(POT_FIELD_COLUMNS)):
                if not (cols >> k) & 1:
                    assert np.all(rows[:, k] == 0.0)
        o.close()


def test_pot_field_consistent_with_energy():
    """The per-atom decomposition carries the energy routine's energies: the
    polarisation energy is 1/2 sum q phi_p, and by symmetry the reaction field
    at the Born ion's centre vanishes next to its potential."""
    o = _born_pair(True)
    e = o.energy()
    rows, pe = o.pot_field(2, 2)
    for k in ("energy_pol", "energy_react", "charge_flux"):
        assert pe[k] == pytest.approx(e[k], rel=1e-12), k
    q = 1.0
    assert 0.5 * q * rows[0, POT_FIELD_COLUMNS.index("phi_p")] == pytest.approx(e["energy_pol"], rel=1e-12)
    # dummies at +-0.001 A carry the ion's Coulomb potential q / (eps_in r)
    eps_in, _, _ = configs.scaled_constants()
    assert rows[1:, 0] == pytest.approx(1.0 / (eps_in * 0.001), rel=1e-9)
    phi_p = abs(rows[0, POT_FIELD_COLUMNS.index("phi_p")])
    ex, ey, ez = np.abs(rows[0, [POT_FIELD_COLUMNS.index(n) for n in ("Ex_p", "Ey_p", "Ez_p")]])
    # the mesh is mirror-symmetric in x and y; z, the axis of the in/out rays,
    # keeps a discretisation-sized asymmetry
    assert max(ex, ey) < 1e-9 * phi_p / 2.0 and ez < 1e-3 * phi_p / 2.0
    o.close()

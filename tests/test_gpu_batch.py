"""The multi-system persistent solve (pbgpu_batch_*): each member's result in
the batch equals its own single-system solve within the solve tolerance, and
the energies agree to 1e-6 relative: a molecule gives the same result alone
and in the mix."""
import numpy as np
import pytest

from cudanextgenpb_b200 import Batch, GpuPath, configs, solver_opts
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu

MOLS = [(60, 7.0, -3.0, 60, 1), (150, 9.0, 2.0, 150, 2), (90, 8.0, 1.0, 91, 1), (40, 6.0, 0.0, 40, 2)]


def _member(spec, group=4):
    na, rad, net, seed, lv = spec
    prob = configs.make_globular_problem(na, rad, net, seed=seed, levels=lv).build()
    g = GpuPath().load(prob)
    g.create_markers()
    g.create_density_map()
    g.assemble(32, 2048, group)
    return prob, g


@pytest.mark.parametrize("precision", ["fp64", "mixed"])
def test_batch_equals_alone(precision):
    members = [_member(s) for s in MOLS]
    opts = solver_opts("cg", tol=1e-10, precision=precision, inner_tol=1e-4, check_every=32)
    alone = []
    for prob, g in members:
        st = g.solve(opts)
        assert st.status == 0
        alone.append((g.phi().copy(), g.energy(), st.iterations))
    b = Batch()
    slots = [b.add(g) for _, g in members]
    stats = b.solve(opts)
    for k, (prob, g) in zip(slots, members):
        st = stats[k]
        assert st.status == 0 and st.rel_residual <= 1e-10, (k, st.status, st.rel_residual)
        phi_a, e_a, it_a = alone[k]
        phi_b = g.phi()
        assert np.linalg.norm(phi_b - phi_a) / np.linalg.norm(phi_a) < 1e-8
        e_b = g.energy()
        assert e_b["sum"] == pytest.approx(e_a["sum"], rel=1e-6)
        if precision == "fp64":
            assert abs(st.iterations - it_a) <= max(3, it_a // 20)
    b.close()
    for _, g in members:
        g.close()


def test_batch_matches_oracle_and_is_deterministic():
    prob, g = _member(MOLS[1])
    o = Oracle(prob)
    o.markers()
    o.density()
    o.assemble()
    ophi, _, _ = o.solve("cg", 1e-12)
    prob2, g2 = _member(MOLS[0])
    b = Batch()
    b.add(g)
    b.add(g2)
    opts = solver_opts("cg", tol=1e-10)
    b.solve(opts)
    phi1 = g.phi().copy()
    assert np.linalg.norm(phi1 - ophi) / np.linalg.norm(ophi) < 1e-6
    b.solve(opts)
    assert np.array_equal(g.phi(), phi1)  # fixed-order reductions: bit-identical reruns
    b.close()


def test_batch_membership_changes():
    members = [_member(s) for s in MOLS[:3]]
    b = Batch()
    slots = [b.add(g) for _, g in members]
    b.remove(slots[1])
    stats = b.solve(solver_opts("cg", tol=1e-9))
    assert set(stats) == {slots[0], slots[2]}
    assert b.add(members[1][1]) == slots[1]  # the freed slot is reused
    stats = b.solve(solver_opts("cg", tol=1e-9))
    assert all(s.status == 0 for s in stats.values())
    b.close()


def test_batch_rejects_unsupported():
    from cudanextgenpb_b200 import PBError
    prob, g = _member(MOLS[0], group=1)
    b = Batch()
    b.add(g)
    with pytest.raises(PBError):
        b.solve(solver_opts("cg", tol=1e-9))  # group 1 layout
    with pytest.raises(PBError):
        b.solve(solver_opts("bicgstab", tol=1e-9))
    b.close()


def test_batch_continuous_membership():
    """Continuous batching: members join a running session at a step boundary
    and leave when done; each result equals the member's own solve."""
    members = [_member(s) for s in MOLS]
    opts = solver_opts("cg", tol=1e-10, precision="mixed", inner_tol=1e-4)
    alone = []
    for _, g in members:
        g.solve(opts)
        alone.append(g.energy()["sum"])
    b = Batch()
    b.set_blocks_per_sm(2)
    b.begin(opts)
    slot_of = {}
    slot_of[0] = b.add(members[0][1])
    slot_of[1] = b.add(members[1][1])
    b.step(40)
    slot_of[2] = b.add(members[2][1])  # joins mid-session
    finished = {}
    for _ in range(400):
        active = b.step(32)
        for j, k in list(slot_of.items()):
            done, st = b.member(k)
            if done:
                assert st.status == 0 and st.rel_residual <= 1e-10
                finished[j] = members[j][1].energy()["sum"]
                b.remove(k)
                del slot_of[j]
                if j == 0:
                    slot_of[3] = b.add(members[3][1])  # takes the freed slot
        if not slot_of:
            break
    assert sorted(finished) == [0, 1, 2, 3]
    for j, e in finished.items():
        assert e == pytest.approx(alone[j], rel=1e-6)
    b.close()


@pytest.mark.parametrize("k", [5, 40])
def test_many_charge_vectors_equal_single_solves(k):
    """pbgpu_solve_charges: k charge vectors on one assembled matrix give, for
    every vector, the energy of a plain solve with those charges."""
    from cudanextgenpb_b200 import solve_charges
    prob, g = _member(MOLS[1])
    pos, q, _ = prob.atoms()
    rng = np.random.default_rng(64)
    Q = np.repeat(q[None, :], k, axis=0)
    for j in range(k):
        sites = rng.choice(len(q), size=8, replace=False)
        Q[j, sites] += rng.choice([-1.0, 1.0], size=8)
    opts = solver_opts("cg", tol=1e-10)
    es, ss = solve_charges(g, Q, opts)
    assert all(s.status == 0 and s.rel_residual <= 1e-10 for s in ss)
    # the context keeps its own charges
    e0, _ = g.run(opts)
    ref0 = GpuPath().load(prob)
    e_ref0, _ = ref0.run(opts)
    assert e0["sum"] == pytest.approx(e_ref0["sum"], rel=1e-9)
    for j in (0, k // 2, k - 1):
        h = GpuPath().load(prob)
        h.set_atoms(pos, Q[j])
        e, st = h.run(opts)
        assert es[j]["sum"] == pytest.approx(e["sum"], rel=1e-6)
        assert abs(ss[j].iterations - st.iterations) <= max(3, st.iterations // 20)
        h.close()
    ref0.close()
    g.close()

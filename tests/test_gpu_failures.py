"""Failure detection on the GPU path, without faulting, trapping or hanging a GPU.

* Admission: a request whose device-memory estimate alone exceeds the server's
  HBM budget is rejected with PBGPU_REJECTED instead of running over budget;
  requests that fit are still served.
* Bounded device-side waits: with the wait limit set to 0 the staged SpMV's
  bulk-copy wait and the persistent kernel's member barrier give up at once;
  the call returns PBGPU_TIMEOUT, and the same context or batch then solves
  normally with the default limit.
* Non-finite input: a NaN charge reaches the right-hand side, and every solver
  reports PBGPU_BREAKDOWN instead of returning a NaN potential as converged.
* The reference's MUMPS option (linear_solver = mumps) through the host
  driver: the direct solve's semantics are a solution to rounding, checked
  against a sparse LU of the oracle's matrix."""
import ctypes as C

import numpy as np
import pytest

from cudanextgenpb_b200 import Batch, GpuPath, PBError, Server, configs, solver_opts
from cudanextgenpb_b200 import _native as N
from oracle_lib import Oracle

pytestmark = pytest.mark.gpu


def _mol(na=60, radius=7.0, net=-3.0, seed=60, levels=1):
    return configs.make_globular_problem(na, radius, net, seed=seed, levels=levels).build()


def _setup(g, group=4):
    g.create_markers()
    g.create_density_map()
    g.assemble(32, 2048, group)


@pytest.mark.parametrize("mode", [0, 1])
def test_server_rejects_request_over_budget(mode):
    small, big = _mol(), _mol(300, 11.0, -3.0, 300, 2)
    ref = GpuPath().load(small)
    e_ref, _ = ref.run(solver_opts("cg", tol=1e-10))
    ref.close()
    probe = Server(tol=1e-10, mode=mode, workers=2)
    need_small = probe.estimate(probe.request(small))
    need_big = probe.estimate(probe.request(big))
    probe.close()
    assert need_big > need_small
    budget = (need_small + need_big) / 2.0  # the small request fits, the big one never can
    srv = Server(tol=1e-10, mode=mode, workers=2, hbm_budget_bytes=budget)
    srv.submit(srv.request(big, tag=1))
    srv.submit(srv.request(small, tag=2))
    results = {}
    for _ in range(20000):
        for r in srv.progress():
            results[r["tag"]] = r
        q, running, _ = srv.pending()
        if len(results) == 2 and q == 0 and running == 0:
            break
    srv.close()
    assert results[1]["status"] == N.PBGPU_REJECTED
    assert results[2]["status"] == 0
    assert results[2]["energy"]["sum"] == pytest.approx(e_ref["sum"], rel=1e-6)


def test_staged_spmv_wait_limit_gives_timeout_and_context_recovers():
    prob = _mol()
    g = GpuPath().load(prob)
    _setup(g, group=1)  # C = 32, G = 1: the SpMV stages slices through bulk async copies
    g.set_wait_limit(0.0)
    with pytest.raises(PBError) as ei:
        g.solve(solver_opts("cg", tol=1e-10))
    assert ei.value.code == N.PBGPU_TIMEOUT
    g.set_wait_limit(1.0)
    st = g.solve(solver_opts("cg", tol=1e-10))
    assert st.status == 0 and st.rel_residual <= 1e-10
    e = g.energy()
    ref = GpuPath().load(prob)
    _setup(ref)
    ref.solve(solver_opts("cg", tol=1e-10))
    assert e["sum"] == pytest.approx(ref.energy()["sum"], rel=1e-9)
    ref.close()
    g.close()


def test_batch_barrier_wait_limit_gives_timeout_and_batch_recovers():
    prob = _mol()
    g = GpuPath().load(prob)
    _setup(g)
    b = Batch()
    b.add(g)
    b.set_wait_limit(0.0)  # the single member owns every resident CTA: the first barrier waits
    with pytest.raises(PBError) as ei:
        b.solve(solver_opts("cg", tol=1e-10))
    assert ei.value.code == N.PBGPU_TIMEOUT
    b.set_wait_limit(2.0)
    st = b.solve(solver_opts("cg", tol=1e-10))[0]
    assert st.status == 0 and st.rel_residual <= 1e-10
    e = g.energy()
    ref = GpuPath().load(prob)
    e_ref, _ = ref.run(solver_opts("cg", tol=1e-10))
    assert e["sum"] == pytest.approx(e_ref["sum"], rel=1e-6)
    b.close()
    ref.close()
    g.close()


@pytest.mark.parametrize("method,precision", [("cg", "fp64"), ("bicgstab", "fp64"), ("cgs", "fp64"),
                                              ("cg", "mixed"), ("bicgstab", "mixed")])
def test_nan_charge_gives_breakdown(method, precision):
    prob = _mol()
    pos, q, _ = prob.atoms()
    q = q.copy()
    q[7] = float("nan")
    g = GpuPath().load(prob)
    g.set_atoms(pos, q)
    _setup(g)
    with pytest.raises(PBError) as ei:
        g.solve(solver_opts(method, tol=1e-10, precision=precision))
    assert ei.value.code == N.PBGPU_BREAKDOWN
    # the context is still usable with finite charges
    q[7] = 0.1
    g.set_atoms(pos, q)
    _setup(g)
    st = g.solve(solver_opts(method, tol=1e-10, precision=precision))
    assert st.status == 0
    g.close()


def test_nan_charge_in_a_batch_gives_breakdown_for_that_member_only():
    prob = _mol()
    pos, q, _ = prob.atoms()
    bad_q = q.copy()
    bad_q[3] = float("nan")
    bad, good = GpuPath().load(prob), GpuPath().load(prob)
    bad.set_atoms(pos, bad_q)
    for g in (bad, good):
        _setup(g)
    b = Batch()
    sb, sg = b.add(bad), b.add(good)
    stats = (N.PbgpuSolveStats * 2)()
    opts = solver_opts("cg", tol=1e-10)
    rc = b._lib.pbgpu_batch_solve(b._b, C.byref(opts), stats)
    assert rc == N.PBGPU_BREAKDOWN
    assert stats[sb].status == N.PBGPU_BREAKDOWN
    assert stats[sg].status == 0 and stats[sg].rel_residual <= 1e-10
    e = good.energy()
    ref = GpuPath().load(prob)
    e_ref, _ = ref.run(solver_opts("cg", tol=1e-10))
    assert e["sum"] == pytest.approx(e_ref["sum"], rel=1e-6)
    ref.close()
    b.close()
    bad.close()
    good.close()


def test_mumps_option_through_host_driver():
    """linear_solver = mumps in options.prm runs the host driver's
    mumps_compute_electric_potential; its solution must equal a direct sparse
    LU solve of the oracle's matrix (the reference's MUMPS semantics)."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    text = configs.born_options().replace("linear_solver = lis", "linear_solver = mumps")
    from cudanextgenpb_b200 import Problem
    prob = Problem(text)
    prob.set_atoms(*configs.BORN_ATOM)
    prob.build()
    e, st = prob.run_gpu()
    assert st.status == 0 and st.iterations > 0 and st.rel_residual <= 1e-12
    o = Oracle(prob)
    o.markers()
    o.density()
    rp, col, val, rhs = o.assemble()
    A = sp.csr_matrix((val, col, rp), shape=(o.n, o.n))
    x = spla.spsolve(A.tocsc(), rhs)
    lib = N.load_gpu()
    ctx = prob._lib.pbhost_gpu_ctx(prob._h)
    phi = np.zeros(o.n)
    assert lib.pbgpu_get_phi(ctx, phi.ctypes.data_as(C.POINTER(C.c_double))) == 0
    assert np.linalg.norm(phi - x) / np.linalg.norm(x) <= 1e-9
    o.set_phi(x)
    oe = o.energy()
    assert e["sum"] == pytest.approx(oe["sum"], rel=1e-9)
    o.close()

"""The continuous-batching server (pbgpu_server_*): requests of different
sizes admitted while others run; each result equals the same molecule solved
alone with the plain FP64 path within 1e-6 relative energy; admission keeps
the held device bytes under the budget."""
import numpy as np
import pytest

from cudanextgenpb_b200 import GpuPath, Server, configs, solver_opts

pytestmark = pytest.mark.gpu

SPECS = [(60, 7.0, -3.0, 60, 1), (150, 9.0, 2.0, 150, 2), (90, 8.0, 1.0, 91, 1), (40, 6.0, 0.0, 40, 2),
         (120, 8.5, -1.0, 120, 1), (200, 10.0, 3.0, 200, 1)]


@pytest.fixture(scope="module")
def pool():
    out = []
    for na, rad, net, seed, lv in SPECS:
        prob = configs.make_globular_problem(na, rad, net, seed=seed, levels=lv).build()
        g = GpuPath().load(prob)
        e, st = g.run(solver_opts("cg", tol=1e-10))
        g.close()
        out.append((prob, e["sum"]))
    return out


@pytest.mark.parametrize("precision,mode", [("mixed", 0), ("fp64", 0), ("mixed", 1), ("fp64", 1)])
def test_server_results_equal_alone(pool, precision, mode):
    srv = Server(tol=1e-10, precision=precision, max_members=3, steps_per_tick=24, mode=mode, workers=3)
    ids = {}
    for k, (prob, _) in enumerate(pool[:3]):
        ids[srv.submit(srv.request(prob, tag=k))] = k
    results = {}
    for tick in range(20000):
        for r in srv.progress():
            results[r["tag"]] = r
        if tick == 2:  # more requests arrive while the first ones run
            for k, (prob, _) in enumerate(pool[3:], start=3):
                ids[srv.submit(srv.request(prob, tag=k))] = k
        q, running, held = srv.pending()
        if len(results) == len(pool) and q == 0 and running == 0:
            break
    assert sorted(results) == list(range(len(pool)))
    for k, r in results.items():
        assert r["status"] == 0 and r["rel_residual"] <= 1e-10
        assert r["energy"]["sum"] == pytest.approx(pool[k][1], rel=1e-6)
        assert r["latency_ms"] >= r["queue_ms"] >= 0
    srv.close()


def test_server_admission_respects_budget(pool):
    prob, _ = pool[1]
    srv = Server(tol=1e-8, max_members=8)
    est = srv.estimate(srv.request(prob))
    srv.close()
    # room for about two of these at a time; the estimate bounds what a
    # context really holds, so the held device bytes stay within the budget
    # (contexts hold less than the estimate, so a third request may fit
    # while another one finishes)
    budget = 2.5 * est
    srv = Server(tol=1e-8, max_members=8, hbm_budget_bytes=budget)
    for k in range(5):
        srv.submit(srv.request(prob, tag=k))
    done = 0
    max_running = 0
    max_held = 0
    for _ in range(5000):
        done += len(srv.progress())
        q, running, held = srv.pending()
        max_running = max(max_running, running)
        max_held = max(max_held, held)
        if done == 5:
            break
    assert done == 5
    assert max_held <= budget
    assert max_running <= 3
    srv.close()


def test_server_charges_on_same_mesh(pool):
    """Requests may carry other charges on the same atoms (titration states)."""
    prob, _ = pool[0]
    pos, q, _ = prob.atoms()
    rng = np.random.default_rng(7)
    srv = Server(tol=1e-10, precision="fp64")
    variants = []
    for k in range(3):
        q2 = q.copy()
        sites = rng.choice(len(q2), size=4, replace=False)
        q2[sites] += rng.choice([-1.0, 1.0], size=4)
        variants.append(q2)
        srv.submit(srv.request(prob, pos, q2, tag=k))
    got = {}
    for _ in range(3000):
        for r in srv.progress():
            got[r["tag"]] = r["energy"]["sum"]
        if len(got) == 3:
            break
    for k, q2 in enumerate(variants):
        g = GpuPath().load(prob)
        g.set_atoms(pos, q2)
        e, _ = g.run(solver_opts("cg", tol=1e-10))
        g.close()
        assert got[k] == pytest.approx(e["sum"], rel=1e-6)
    srv.close()


@pytest.mark.parametrize("mode", [0, 1])
def test_server_builds_request_meshes(pool, mode):
    """Requests that carry only the molecule (atoms, options): the server
    builds each mesh on the GPU (initial octree, surface refinement, nodes,
    rays) as the first step of serving it; results equal the host-meshed
    plain solves."""
    srv = Server(tol=1e-10, precision="mixed", max_members=3, steps_per_tick=24, mode=mode, workers=3)
    probs = []
    for k, (na, rad, net, seed, lv) in enumerate(SPECS):
        p = configs.make_globular_problem(na, rad, net, seed=seed, levels=lv)
        b = p.mesh_build()
        probs.append((p, b))
        srv.submit(srv.request(p, tag=k, build=b))
    results = {}
    for _ in range(20000):
        for r in srv.progress():
            results[r["tag"]] = r
        q, running, _ = srv.pending()
        if len(results) == len(SPECS) and q == 0 and running == 0:
            break
    srv.close()
    assert sorted(results) == list(range(len(SPECS)))
    for k, r in results.items():
        assert r["status"] == 0 and r["rel_residual"] <= 1e-10
        assert r["energy"]["sum"] == pytest.approx(pool[k][1], rel=1e-6)


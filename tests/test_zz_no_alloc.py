"""pbgpu_coulomb_energy_static, the Coulomb energy for callers that cannot
allocate device memory (code inside another library's enqueue or plugin
callback, or a process whose device memory belongs to a pool allocator).

Its result is checked against the Coulomb term of pbgpu_energy, the existing
entry point, on two calls in a row: the fixed scratch keeps the previous call's
contents, and the second call must not depend on them.  Device buffers come from
torch, so the test itself allocates nothing through the library.  The cases
cover the tiny inputs (0 and 1 atoms: a zero written on the stream without
waiting), atoms whose charge is below the reference's threshold (one of them on
top of a charged atom), a grid of many blocks whose partials the last block
sums, and a torch side stream instead of the default one."""
import ctypes

import numpy as np
import pytest

from cudanextgenpb_b200 import GpuPath, configs, solver_opts
from cudanextgenpb_b200 import _native as N

pytestmark = pytest.mark.gpu


def _static(lib, atoms_dev, n, e_in, T, out, stream):
    return lib.pbgpu_coulomb_energy_static(ctypes.c_void_p(atoms_dev.data_ptr()), n, e_in, T,
                                           ctypes.c_void_p(out.data_ptr()), ctypes.c_void_p(stream.cuda_stream))


def _two_calls(atoms_np, e_in, T, side_stream):
    """Two calls in a row on a torch stream; returns both values."""
    import torch

    dev = torch.tensor(atoms_np.reshape(-1), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    lib = N.load_gpu()
    stream = torch.cuda.Stream() if side_stream else torch.cuda.current_stream()
    values = []
    for _ in range(2):
        with torch.cuda.stream(stream):
            out.fill_(float("nan"))
            st = _static(lib, dev, atoms_np.shape[0], e_in, T, out, stream)
            assert st == 0
        stream.synchronize()
        values.append(out.item())
    return values


@pytest.mark.parametrize("n_atoms,radius,seed,levels,side", [(60, 7.0, 60, 1, False), (300, 11.0, 300, 1, True)])
def test_static_coulomb_matches_energy_entry_point(n_atoms, radius, seed, levels, side):
    prob = configs.make_globular_problem(n_atoms, radius, -3.0, seed=seed, levels=levels).build()
    g = GpuPath().load(prob)
    e, _ = g.run(solver_opts("cg", tol=1e-8))
    ref = e["energy_coul"]
    assert ref != 0.0
    g.close()
    pos, q, _ = prob.atoms()
    model = prob.model()
    for v in _two_calls(np.concatenate([pos, q[:, None]], axis=1), model.e_in, model.T, side):
        assert v == pytest.approx(ref, rel=1e-12)


def test_static_coulomb_uncharged_atoms_match_energy_entry_point():
    """Atoms with |q| <= 1e-5 drop out, as in pbgpu_energy; a zero-charge atom
    placed exactly on a charged one must not turn the sum into NaN."""
    prob = configs.make_globular_problem(60, 7.0, -3.0, seed=61, levels=1).build()
    pos, q, _ = prob.atoms()
    q = q.copy()
    q[::7] = 0.0
    q[3] = 4e-6
    q[5] = -9e-6
    pos = np.concatenate([pos, pos[1:2]], axis=0)  # an uncharged atom on top of atom 1 (charged)
    q = np.concatenate([q, [0.0]])
    assert q[1] != 0.0
    g = GpuPath().load(prob)
    g.set_atoms(pos, q)
    e, _ = g.run(solver_opts("cg", tol=1e-8))
    ref = e["energy_coul"]
    g.close()
    assert np.isfinite(ref) and ref != 0.0
    model = prob.model()
    for v in _two_calls(np.concatenate([pos, q[:, None]], axis=1), model.e_in, model.T, True):
        assert np.isfinite(v)
        assert v == pytest.approx(ref, rel=1e-12)


@pytest.mark.parametrize("n", [0, 1])
def test_static_coulomb_fewer_than_two_atoms(n):
    """No pair: zero, written on the (side) stream over whatever the output held."""
    atoms = np.array([[1.0, 2.0, 3.0, 0.7]] * max(n, 1))[:max(n, 1)]
    for v in _two_calls(atoms, 2.0, 298.15, True):
        assert v == 0.0


def test_static_coulomb_many_rows():
    """20,000 atoms: 79 blocks of 256 rows, each row tile meeting up to 79 atom
    tiles, and the last block to finish summing 79 partials.  The reference
    value is a float64 numpy pair sum in the same units."""
    rng = np.random.default_rng(20000)
    n = 20000
    pos = rng.uniform(-60.0, 60.0, size=(n, 3))
    q = rng.normal(0.0, 0.35, size=n)
    q[rng.integers(0, n, size=200)] = 0.0
    e_in, T = 2.0, 298.15
    e_0, kb, e, angs = 8.85418781762e-12, 1.380649e-23, 1.602176634e-19, 1e-10
    eps_in = 4.0 * np.pi * e_0 * e_in * kb * T * angs / (e * e)
    qq = np.where(np.abs(q) > 1e-5, q, 0.0)
    total = 0.0
    for i in range(0, n, 500):  # row blocks of the upper triangle
        d = np.linalg.norm(pos[i:i + 500, None, :] - pos[None, :, :], axis=2)
        mask = np.arange(n)[None, :] > np.arange(i, min(i + 500, n))[:, None]
        inv = np.where(mask, 1.0 / np.where(mask, d, 1.0), 0.0)
        total += float(qq[i:i + 500] @ inv @ qq)
    ref = total / eps_in
    for v in _two_calls(np.concatenate([pos, q[:, None]], axis=1), e_in, T, True):
        assert v == pytest.approx(ref, rel=1e-10)


def test_static_coulomb_rejects_oversize():
    import torch

    lib = N.load_gpu()
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = lib.pbgpu_coulomb_energy_static(ctypes.c_void_p(buf.data_ptr()), 131073, 2.0, 298.15,
                                         ctypes.c_void_p(out.data_ptr()), None)
    assert st == N.PBGPU_ERR_CAPACITY

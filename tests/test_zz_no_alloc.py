"""pbgpu_coulomb_energy_static, the Coulomb energy for callers that cannot
allocate device memory (code inside another library's enqueue or plugin
callback, or a process whose device memory belongs to a pool allocator).

Its result is checked against the Coulomb term of pbgpu_energy, the existing
entry point, on two calls in a row: the fixed scratch keeps the previous call's
contents, and the second call must not depend on them.  Device buffers come from
torch, so the test itself allocates nothing through the library."""
import ctypes

import numpy as np
import pytest

from cudanextgenpb_b200 import GpuPath, configs, solver_opts
from cudanextgenpb_b200 import _native as N

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("n_atoms,radius,seed,levels", [(60, 7.0, 60, 1), (300, 11.0, 300, 1)])
def test_static_coulomb_matches_energy_entry_point(n_atoms, radius, seed, levels):
    import torch

    prob = configs.make_globular_problem(n_atoms, radius, -3.0, seed=seed, levels=levels).build()
    g = GpuPath().load(prob)
    e, _ = g.run(solver_opts("cg", tol=1e-8))
    ref = e["energy_coul"]
    assert ref != 0.0
    g.close()

    pos, q, _ = prob.atoms()
    model = prob.model()
    atoms = torch.tensor(np.concatenate([pos, q[:, None]], axis=1).reshape(-1), dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    lib = N.load_gpu()
    stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
    values = []
    for _ in range(2):
        out.fill_(float("nan"))
        st = lib.pbgpu_coulomb_energy_static(ctypes.c_void_p(atoms.data_ptr()), len(q), model.e_in, model.T,
                                             ctypes.c_void_p(out.data_ptr()), stream)
        assert st == 0
        torch.cuda.synchronize()
        values.append(out.item())
    for v in values:
        assert v == pytest.approx(ref, rel=1e-12)


def test_static_coulomb_rejects_oversize():
    import torch

    lib = N.load_gpu()
    buf = torch.zeros(4, dtype=torch.float64, device="cuda")
    out = torch.zeros(1, dtype=torch.float64, device="cuda")
    st = lib.pbgpu_coulomb_energy_static(ctypes.c_void_p(buf.data_ptr()), 131073, 2.0, 298.15,
                                         ctypes.c_void_p(out.data_ptr()), None)
    assert st == N.PBGPU_ERR_CAPACITY

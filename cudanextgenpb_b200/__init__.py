"""B200-native (sm_100a) assemble / solve / energy path for NextGenPB's
linearized Poisson-Boltzmann model on 2:1-balanced octrees.

Native pieces (built in-tree by ``cudanextgenpb_b200.build``):
  lib/libpbgpu.so   the GPU path behind the C ABI of include/pbgpu.h
  lib/libpbhost.so  the host poisson_boltzmann mirror (include/pbhost.h)
"""
from .pb import Batch, GpuPath, PBError, Problem, Server, parse_lis_options, solve_charges, solver_opts  # noqa: F401

__all__ = ["GpuPath", "PBError", "Problem", "parse_lis_options", "solver_opts"]

"""ctypes bindings of the two native libraries built in-tree.

``libpbgpu.so`` exposes the C ABI of include/pbgpu.h (the GPU path),
``libpbhost.so`` the C API of include/pbhost.h (options, atoms, octree and
surface rays).  Loading fails loudly when a library is missing: there is no
fallback implementation.
"""
from __future__ import annotations

import ctypes as C
import os

LIB_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "lib")

i32, i64, u64, dbl = C.c_int32, C.c_int64, C.c_uint64, C.c_double
P = C.POINTER


class PbgpuMesh(C.Structure):
    _fields_ = [("n_oct", i64), ("oct_xyz", P(i32)), ("oct_level", P(C.c_int8)), ("oct_nodes", P(i32)),
                ("n_nodes", i64), ("node_xyz", P(i32)), ("n_hang", i64), ("hang_np", P(C.c_int8)),
                ("hang_par", P(i32)), ("lo", dbl * 3), ("hi", dbl * 3), ("locate_tol", dbl)]


class PbgpuRays(C.Structure):
    _fields_ = [("n_rays", i64), ("keys", P(u64)), ("ptr", P(i64)), ("inters", P(dbl)), ("normals", P(dbl))]


class PbgpuModel(C.Structure):
    _fields_ = [("e_in", dbl), ("e_out", dbl), ("ionic_strength", dbl), ("T", dbl), ("bc_type", C.c_int),
                ("stern_layer_surf", C.c_int), ("stern_layer", dbl), ("calc_energy", C.c_int),
                ("calc_coulombic", C.c_int)]


class PbgpuSellOpts(C.Structure):
    _fields_ = [("chunk", C.c_int), ("sigma", C.c_int), ("group", C.c_int)]


class PbgpuSolverOpts(C.Structure):
    _fields_ = [("method", C.c_int), ("precond", C.c_int), ("precision", C.c_int), ("tol", dbl),
                ("max_iter", C.c_int), ("inner_tol", dbl), ("max_outer", C.c_int), ("check_every", C.c_int),
                ("conv_cond", C.c_int), ("tol_w", dbl)]


class PbgpuSolveStats(C.Structure):
    _fields_ = [("status", C.c_int), ("iterations", C.c_int), ("outer", C.c_int), ("rel_residual", dbl),
                ("device_ms", dbl)]


class PbgpuEnergyOut(C.Structure):
    _fields_ = [("energy_pol", dbl), ("energy_react", dbl), ("energy_coul", dbl), ("charge_flux", dbl),
                ("net_charge", dbl), ("sum", dbl)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_}


class PbgpuPotFieldOut(C.Structure):
    _fields_ = [("energy_pol", dbl), ("energy_react", dbl), ("energy_coul", dbl), ("charge_flux", dbl),
                ("columns", C.c_int), ("reserved", C.c_int)]

    def as_dict(self):
        return {k: getattr(self, k) for k, _ in self._fields_ if k != "reserved"}


# pot_field.dat column names in the order of the per-atom rows
POT_FIELD_COLUMNS = ("phi_c", "phi_p", "phi_i", "Ex_c", "Ey_c", "Ez_c", "Ex_p", "Ey_p", "Ez_p",
                     "Ex_i", "Ey_i", "Ez_i")


class PbgpuCounters(C.Structure):
    _fields_ = [("launches", i64), ("spmv_launches", i64), ("spmv_ms", dbl), ("spmv_bytes", dbl),
                ("krylov_iterations", i64), ("energy_points", i64), ("energy_pairs", i64),
                ("device_bytes", i64)]


class PbgpuMeshBuild(C.Structure):
    _fields_ = [("n_oct", i64), ("oct_xyz", P(i32)), ("oct_level", P(C.c_int8)), ("lo", dbl * 3), ("hi", dbl * 3),
                ("locate_tol", dbl), ("refine", C.c_int), ("minlevel", C.c_int), ("maxlevel", C.c_int),
                ("unilevel", C.c_int), ("n_spheres", i64), ("spheres", P(dbl)), ("init_level", C.c_int),
                ("box_level", C.c_int), ("box_lo", dbl * 3), ("box_hi", dbl * 3)]


class PbgpuRequest(C.Structure):
    _fields_ = [("mesh", P(PbgpuMesh)), ("rays", PbgpuRays * 3), ("n_atoms", i64), ("pos", P(dbl)),
                ("charge", P(dbl)), ("model", P(PbgpuModel)), ("user_tag", i64), ("build", P(PbgpuMeshBuild))]


class PbgpuResult(C.Structure):
    _fields_ = [("id", i64), ("user_tag", i64), ("status", C.c_int), ("energy", PbgpuEnergyOut),
                ("stats", PbgpuSolveStats), ("latency_ms", dbl), ("queue_ms", dbl)]


class PbgpuServerOpts(C.Structure):
    _fields_ = [("hbm_budget_bytes", dbl), ("max_members", C.c_int), ("steps_per_tick", C.c_int),
                ("blocks_per_sm", C.c_int), ("solver", PbgpuSolverOpts), ("energy_fast", C.c_int),
                ("admit_per_tick", C.c_int), ("mode", C.c_int), ("workers", C.c_int)]


class PbhostInfo(C.Structure):
    _fields_ = [("mesh_shape", C.c_int), ("unilevel", C.c_int), ("minlevel", C.c_int), ("maxlevel", C.c_int),
                ("outlevel", C.c_int), ("scale_level", C.c_int), ("loc_refinement", C.c_int), ("scale", dbl),
                ("lo", dbl * 3), ("hi", dbl * 3), ("cc", dbl * 3), ("l_c", dbl * 3), ("r_c", dbl * 3),
                ("l_cr", dbl * 3), ("r_cr", dbl * 3), ("pot_bc", dbl), ("locate_tol", dbl), ("n_oct", i64),
                ("n_nodes", i64), ("n_hang", i64), ("n_atoms", i64), ("n_rays", i64 * 3), ("net_charge", dbl)]


PBGPU_OK = 0
PBGPU_ERR_ARG, PBGPU_ERR_CUDA, PBGPU_ERR_OOM, PBGPU_ERR_STATE, PBGPU_ERR_CAPACITY = 1, 2, 3, 4, 5
PBGPU_NOT_CONVERGED, PBGPU_BREAKDOWN, PBGPU_TIMEOUT, PBGPU_REJECTED = 10, 11, 12, 13
PBGPU_CG, PBGPU_BICGSTAB, PBGPU_CGS = 0, 1, 2
PBGPU_PRECOND_NONE, PBGPU_PRECOND_JACOBI, PBGPU_PRECOND_BLOCK_JACOBI = 0, 1, 2
PBGPU_FP64, PBGPU_MIXED = 0, 1

ctx_p = C.c_void_p

# name -> (restype, argtypes); every symbol include/pbgpu.h declares
PBGPU_FUNCS = {
    "pbgpu_version": (C.c_int, []),
    "pbgpu_ctx_create": (C.c_int, [P(ctx_p), C.c_int, C.c_void_p]),
    "pbgpu_ctx_destroy": (None, [ctx_p]),
    "pbgpu_last_error": (C.c_char_p, [ctx_p]),
    "pbgpu_ctx_stream": (C.c_void_p, [ctx_p]),
    "pbgpu_set_mesh": (C.c_int, [ctx_p, P(PbgpuMesh)]),
    "pbgpu_set_rays": (C.c_int, [ctx_p, C.c_int, P(PbgpuRays)]),
    "pbgpu_set_atoms": (C.c_int, [ctx_p, i64, P(dbl), P(dbl)]),
    "pbgpu_set_model": (C.c_int, [ctx_p, P(PbgpuModel)]),
    "pbgpu_create_markers": (C.c_int, [ctx_p]),
    "pbgpu_create_density_map": (C.c_int, [ctx_p]),
    "pbgpu_assemble": (C.c_int, [ctx_p, P(PbgpuSellOpts)]),
    "pbgpu_solve": (C.c_int, [ctx_p, P(PbgpuSolverOpts), P(PbgpuSolveStats)]),
    "pbgpu_phi_on_atoms": (C.c_int, [ctx_p, P(dbl)]),
    "pbgpu_energy": (C.c_int, [ctx_p, C.c_int, P(PbgpuEnergyOut)]),
    "pbgpu_pot_field": (C.c_int, [ctx_p, C.c_int, C.c_int, C.c_int, P(dbl), P(PbgpuPotFieldOut)]),
    "pbgpu_parse_lis_options": (C.c_int, [C.c_char_p, P(PbgpuSolverOpts)]),
    "pbgpu_default_solver_opts": (None, [P(PbgpuSolverOpts)]),
    "pbgpu_get_node_coeffs": (C.c_int, [ctx_p, P(dbl), P(dbl)]),
    "pbgpu_get_markers": (C.c_int, [ctx_p, P(dbl), P(i64), P(i32)]),
    "pbgpu_get_fractions": (C.c_int, [ctx_p, P(dbl)]),
    "pbgpu_get_density": (C.c_int, [ctx_p, P(dbl), P(dbl)]),
    "pbgpu_get_system": (C.c_int, [ctx_p, P(i64), P(i64), P(i32), P(dbl), P(dbl)]),
    "pbgpu_get_phi": (C.c_int, [ctx_p, P(dbl)]),
    "pbgpu_get_stage_ms": (C.c_int, [ctx_p, P(dbl)]),
    "pbgpu_set_profiling": (C.c_int, [ctx_p, C.c_int]),
    "pbgpu_set_wait_limit": (C.c_int, [ctx_p, dbl]),
    "pbgpu_get_counters": (C.c_int, [ctx_p, P(PbgpuCounters)]),
    "pbgpu_reset_counters": (C.c_int, [ctx_p]),
    "pbgpu_coulomb_energy_static": (C.c_int, [C.c_void_p, i64, dbl, dbl, C.c_void_p, C.c_void_p]),
    "pbgpu_autotune": (C.c_int, [ctx_p, C.c_int, P(PbgpuSellOpts), P(C.c_int), P(dbl)]),
    "pbgpu_build_mesh": (C.c_int, [ctx_p, P(PbgpuMeshBuild)]),
    "pbgpu_get_mesh_counts": (C.c_int, [ctx_p, P(i64), P(i64), P(i64), P(i64)]),
    "pbgpu_get_mesh": (C.c_int, [ctx_p, P(C.c_int32), P(C.c_int8), P(C.c_int32), P(C.c_int32), P(C.c_int8),
                                 P(C.c_int32), P(dbl)]),
    "pbgpu_solve_charges": (C.c_int, [ctx_p, C.c_int, P(dbl), P(PbgpuSolverOpts), C.c_int, P(PbgpuEnergyOut),
                                      P(PbgpuSolveStats)]),
    "pbgpu_batch_create": (C.c_int, [P(C.c_void_p), C.c_int, C.c_void_p]),
    "pbgpu_batch_destroy": (None, [C.c_void_p]),
    "pbgpu_batch_last_error": (C.c_char_p, [C.c_void_p]),
    "pbgpu_batch_add": (C.c_int, [C.c_void_p, ctx_p, P(C.c_int)]),
    "pbgpu_batch_remove": (C.c_int, [C.c_void_p, C.c_int]),
    "pbgpu_batch_size": (C.c_int, [C.c_void_p]),
    "pbgpu_batch_solve": (C.c_int, [C.c_void_p, P(PbgpuSolverOpts), P(PbgpuSolveStats)]),
    "pbgpu_batch_begin": (C.c_int, [C.c_void_p, P(PbgpuSolverOpts)]),
    "pbgpu_batch_step": (C.c_int, [C.c_void_p, C.c_int, P(C.c_int)]),
    "pbgpu_batch_member": (C.c_int, [C.c_void_p, C.c_int, P(C.c_int), P(PbgpuSolveStats)]),
    "pbgpu_batch_set_blocks_per_sm": (C.c_int, [C.c_void_p, C.c_int]),
    "pbgpu_batch_set_wait_limit": (C.c_int, [C.c_void_p, dbl]),
    "pbgpu_batch_launch": (C.c_int, [C.c_void_p, C.c_int]),
    "pbgpu_batch_wait": (C.c_int, [C.c_void_p, P(C.c_int)]),
    "pbgpu_default_server_opts": (None, [P(PbgpuServerOpts)]),
    "pbgpu_server_create": (C.c_int, [P(C.c_void_p), C.c_int, P(PbgpuServerOpts)]),
    "pbgpu_server_destroy": (None, [C.c_void_p]),
    "pbgpu_server_last_error": (C.c_char_p, [C.c_void_p]),
    "pbgpu_server_submit": (C.c_int, [C.c_void_p, P(PbgpuRequest), P(i64)]),
    "pbgpu_server_progress": (C.c_int, [C.c_void_p, P(PbgpuResult), C.c_int, P(C.c_int)]),
    "pbgpu_server_pending": (C.c_int, [C.c_void_p, P(C.c_int), P(C.c_int), P(i64)]),
    "pbgpu_server_stats": (C.c_int, [C.c_void_p, P(i64), P(i64), P(i64), P(i64)]),
    "pbgpu_request_bytes_estimate": (i64, [P(PbgpuRequest)]),
}

host_p = C.c_void_p
PBHOST_FUNCS = {
    "pbhost_create": (host_p, []),
    "pbhost_destroy": (None, [host_p]),
    "pbhost_last_error": (C.c_char_p, [host_p]),
    "pbhost_load_options_file": (C.c_int, [host_p, C.c_char_p]),
    "pbhost_load_options_text": (C.c_int, [host_p, C.c_char_p]),
    "pbhost_set_option": (C.c_int, [host_p, C.c_char_p, C.c_char_p]),
    "pbhost_read_pqr": (C.c_int, [host_p, C.c_char_p]),
    "pbhost_set_atoms": (C.c_int, [host_p, i64, P(dbl), P(dbl), P(dbl)]),
    "pbhost_build_problem": (C.c_int, [host_p]),
    "pbhost_build_on_gpu": (C.c_int, [host_p, C.c_void_p]),
    "pbhost_initial_octree": (C.c_int, [host_p, C.c_int, P(PbgpuMeshBuild)]),
    "pbhost_write_vtu": (C.c_int, [host_p, C.c_char_p, C.c_char_p, P(dbl)]),
    "pbhost_get_info": (C.c_int, [host_p, P(PbhostInfo)]),
    "pbhost_get_mesh": (C.c_int, [host_p, P(PbgpuMesh)]),
    "pbhost_get_rays": (C.c_int, [host_p, C.c_int, P(PbgpuRays)]),
    "pbhost_get_atoms": (C.c_int, [host_p, P(dbl), P(dbl), P(dbl)]),
    "pbhost_get_model": (C.c_int, [host_p, P(PbgpuModel)]),
    "pbhost_get_solver_opts": (C.c_int, [host_p, P(PbgpuSolverOpts)]),
    "pbhost_run_gpu": (C.c_int, [host_p, P(PbgpuEnergyOut), P(PbgpuSolveStats)]),
    "pbhost_gpu_ctx": (ctx_p, [host_p]),
}

_gpu = None
_host = None


def _declare(lib, table):
    for name, (res, args) in table.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


def lib_path(name):
    return os.path.join(LIB_DIR, name)


def load_gpu():
    """libpbgpu.so; raises if it has not been built."""
    global _gpu
    if _gpu is None:
        path = lib_path("libpbgpu.so")
        if not os.path.exists(path):
            raise RuntimeError("libpbgpu.so is not built (run __graft_entry__.build())")
        _gpu = _declare(C.CDLL(path, mode=C.RTLD_GLOBAL), PBGPU_FUNCS)
    return _gpu


def load_host():
    global _host
    if _host is None:
        load_gpu()
        path = lib_path("libpbhost.so")
        if not os.path.exists(path):
            raise RuntimeError("libpbhost.so is not built (run __graft_entry__.build())")
        _host = _declare(C.CDLL(path), PBHOST_FUNCS)
    return _host

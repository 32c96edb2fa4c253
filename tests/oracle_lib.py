"""ctypes access to the CPU oracle (oracle/lib/liboracle.so) — test infrastructure.

Only tests, __graft_entry__.smoke() and bench.py's CPU baseline use this.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

from cudanextgenpb_b200 import _native as N

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
ORACLE_SO = os.path.join(ROOT, "oracle", "lib", "liboracle.so")

P = C.POINTER
_lib = None


def load():
    global _lib
    if _lib is None:
        if not os.path.exists(ORACLE_SO):
            raise RuntimeError("oracle not built: run __graft_entry__.build()")
        L = C.CDLL(ORACLE_SO)
        sp = C.c_void_p
        L.oracle_create.restype = sp
        L.oracle_create.argtypes = [P(N.PbgpuMesh), P(N.PbgpuRays), C.c_int64, P(C.c_double), P(C.c_double),
                                    P(N.PbgpuModel)]
        L.oracle_destroy.argtypes = [sp]
        for f in ("oracle_markers", "oracle_density", "oracle_assemble"):
            getattr(L, f).argtypes = [sp]
        L.oracle_assemble_mode.argtypes = [sp, C.c_int]
        L.oracle_solve.argtypes = [sp, C.c_int, C.c_double, C.c_int, C.c_int, P(C.c_double)]
        L.oracle_solve_ex.argtypes = [sp, C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_int, C.c_int,
                                      P(C.c_double)]
        L.oracle_phi_on_atoms.argtypes = [sp, P(C.c_double)]
        L.oracle_energy.argtypes = [sp, C.c_int, P(N.PbgpuEnergyOut)]
        L.oracle_pot_field.argtypes = [sp, C.c_int, C.c_int, C.c_int, P(C.c_double), P(N.PbgpuPotFieldOut)]
        L.oracle_get_node_coeffs.argtypes = [sp, P(C.c_double), P(C.c_double)]
        L.oracle_get_markers.argtypes = [sp, P(C.c_double), P(C.c_int64), P(C.c_int32)]
        L.oracle_get_fractions.argtypes = [sp, P(C.c_double)]
        L.oracle_get_density.argtypes = [sp, P(C.c_double), P(C.c_double)]
        L.oracle_get_system.argtypes = [sp, P(C.c_int64), P(C.c_int64), P(C.c_int32), P(C.c_double), P(C.c_double)]
        L.oracle_get_phi.argtypes = [sp, P(C.c_double)]
        L.oracle_set_phi.argtypes = [sp, P(C.c_double)]
        L.oracle_set_system.argtypes = [sp, C.c_int64, P(C.c_int64), P(C.c_int32), P(C.c_double), P(C.c_double)]
        L.oracle_spmv.argtypes = [sp, P(C.c_double), P(C.c_double), C.c_int]
        L.oracle_tri_table.argtypes = [P(C.c_int)]
        L.oracle_time_cg_iterations.restype = C.c_double
        L.oracle_time_cg_iterations.argtypes = [sp, C.c_int, C.c_int]
        _lib = L
    return _lib


def _d(a):
    return a.ctypes.data_as(P(C.c_double))


class Oracle:
    """The CPU restatement of the reference path on one problem's inputs."""

    def __init__(self, prob, atoms=None):
        """atoms: (pos, q) to use instead of the problem's own."""
        self.L = load()
        m = prob.mesh_struct()
        rays = (N.PbgpuRays * 3)(*[prob.rays_struct(a) for a in range(3)])
        if atoms is None:
            pos, q, _ = prob.atoms()
        else:
            pos, q = np.asarray(atoms[0], dtype=np.float64).reshape(-1, 3), np.asarray(atoms[1], dtype=np.float64)
        self.pos, self.q = np.ascontiguousarray(pos), np.ascontiguousarray(q)
        md = prob.model()
        self.s = self.L.oracle_create(C.byref(m), rays, len(q), _d(self.pos), _d(self.q), C.byref(md))
        if not self.s:
            raise RuntimeError("oracle_create failed")
        self.n, self.n_oct, self.na = m.n_nodes, m.n_oct, len(q)

    def close(self):
        if self.s:
            self.L.oracle_destroy(self.s)
            self.s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def _ok(self, st):
        if st != 0:
            raise RuntimeError("oracle status %d" % st)

    def markers(self):
        self._ok(self.L.oracle_markers(self.s))
        marker = np.zeros(self.n_oct)
        nb = C.c_int64()
        self._ok(self.L.oracle_get_markers(self.s, _d(marker), C.byref(nb), None))
        border = np.zeros(nb.value, dtype=np.int32)
        self._ok(self.L.oracle_get_markers(self.s, None, C.byref(nb), border.ctypes.data_as(P(C.c_int32))))
        return marker, border

    def node_coeffs(self):
        e, r = np.zeros(self.n), np.zeros(self.n)
        self._ok(self.L.oracle_get_node_coeffs(self.s, _d(e), _d(r)))
        return e, r

    def fractions(self, nb):
        f = np.zeros(12 * nb)
        self._ok(self.L.oracle_get_fractions(self.s, _d(f)))
        return f.reshape(-1, 12)

    def density(self):
        self._ok(self.L.oracle_density(self.s))
        rho, vp = np.zeros(self.n), np.zeros(self.n)
        self._ok(self.L.oracle_get_density(self.s, _d(rho), _d(vp)))
        return rho, vp

    def assemble(self, mode=None):
        """mode None: automatic; "triplets" or "rows" forces one assembly."""
        if mode is None:
            self._ok(self.L.oracle_assemble(self.s))
        else:
            self._ok(self.L.oracle_assemble_mode(self.s, 1 if mode == "rows" else 0))
        return self.system()

    def system(self):
        nnz = C.c_int64()
        self._ok(self.L.oracle_get_system(self.s, C.byref(nnz), None, None, None, None))
        rp = np.zeros(self.n + 1, dtype=np.int64)
        col = np.zeros(nnz.value, dtype=np.int32)
        val = np.zeros(nnz.value)
        rhs = np.zeros(self.n)
        self._ok(self.L.oracle_get_system(self.s, None, rp.ctypes.data_as(P(C.c_int64)),
                                          col.ctypes.data_as(P(C.c_int32)), _d(val), _d(rhs)))
        return rp, col, val, rhs

    def set_system(self, rp, col, val, rhs):
        rp = np.ascontiguousarray(rp, dtype=np.int64)
        col = np.ascontiguousarray(col, dtype=np.int32)
        val = np.ascontiguousarray(val, dtype=np.float64)
        rhs = np.ascontiguousarray(rhs, dtype=np.float64)
        self._ok(self.L.oracle_set_system(self.s, self.n, rp.ctypes.data_as(P(C.c_int64)),
                                          col.ctypes.data_as(P(C.c_int32)), _d(val), _d(rhs)))

    def solve(self, method="cg", tol=1e-12, max_iter=100000, threads=0, precond="jacobi", conv_cond=0, tol_w=1.0):
        rel = C.c_double()
        pc = {"none": N.PBGPU_PRECOND_NONE, "jacobi": N.PBGPU_PRECOND_JACOBI,
              "block_jacobi": N.PBGPU_PRECOND_BLOCK_JACOBI}[precond]
        m = {"cg": N.PBGPU_CG, "bicgstab": N.PBGPU_BICGSTAB, "cgs": N.PBGPU_CGS}[method]
        it = self.L.oracle_solve_ex(self.s, m, pc, conv_cond, tol, tol_w, max_iter, threads, C.byref(rel))
        if it < 0:
            raise RuntimeError("oracle_solve failed")
        phi = np.zeros(self.n)
        self._ok(self.L.oracle_get_phi(self.s, _d(phi)))
        return phi, it, rel.value

    def set_phi(self, phi):
        phi = np.ascontiguousarray(phi, dtype=np.float64)
        self._ok(self.L.oracle_set_phi(self.s, _d(phi)))

    def phi_on_atoms(self):
        out = np.zeros(self.na)
        self._ok(self.L.oracle_phi_on_atoms(self.s, _d(out)))
        return out

    def energy(self, fast=False):
        e = N.PbgpuEnergyOut()
        self._ok(self.L.oracle_energy(self.s, 1 if fast else 0, C.byref(e)))
        return e.as_dict()

    def pot_field(self, calc_potential_terms, calc_field_terms, fast=False):
        rows = np.zeros((self.na, len(N.POT_FIELD_COLUMNS)))
        o = N.PbgpuPotFieldOut()
        self._ok(self.L.oracle_pot_field(self.s, 1 if fast else 0, int(calc_potential_terms),
                                         int(calc_field_terms), _d(rows), C.byref(o)))
        return rows, o.as_dict()

    def spmv(self, x, threads=0):
        x = np.ascontiguousarray(x, dtype=np.float64)
        y = np.zeros(self.n)
        self._ok(self.L.oracle_spmv(self.s, _d(x), _d(y), threads))
        return y

    def time_cg(self, iters, threads=0):
        return self.L.oracle_time_cg_iterations(self.s, iters, threads)

    def run(self, method="cg", tol=1e-12, fast=False):
        """markers -> density -> assemble -> solve -> energy."""
        self.markers()
        self.density()
        self.assemble()
        phi, it, rel = self.solve(method, tol)
        return self.energy(fast), phi, it, rel


def problem_arrays(prob) -> dict:
    """A built host problem's oracle inputs as plain numpy arrays (mesh, rays of
    the three axes, atoms, model), for saving and for ArrayProblem."""
    m = prob.mesh()
    d = {"mesh_" + k: np.asarray(v) for k, v in m.items()}
    for a in range(3):
        r = prob.rays(a)
        for k, v in r.items():
            d["rays%d_%s" % (a, k)] = np.asarray(v)
    pos, q, rad = prob.atoms()
    d["atoms_pos"], d["atoms_q"] = pos, q
    md = prob.model()
    d["model"] = np.array([getattr(md, k) for k, _ in md._fields_], dtype=np.float64)
    return d


class ArrayProblem:
    """The inputs Oracle takes (mesh_struct, rays_struct, atoms, model), from
    the arrays of problem_arrays, with no native library besides the oracle."""

    def __init__(self, d):
        self.d = {k: np.ascontiguousarray(v) for k, v in d.items()}

    def _p(self, key, ct):
        return self.d[key].ctypes.data_as(P(ct))

    def mesh_struct(self):
        d = self.d
        m = N.PbgpuMesh()
        m.n_oct, m.n_nodes, m.n_hang = int(d["mesh_n_oct"]), int(d["mesh_n_nodes"]), int(d["mesh_n_hang"])
        m.oct_xyz = self._p("mesh_oct_xyz", C.c_int32)
        m.oct_level = self._p("mesh_oct_level", C.c_int8)
        m.oct_nodes = self._p("mesh_oct_nodes", C.c_int32)
        m.node_xyz = self._p("mesh_node_xyz", C.c_int32)
        if m.n_hang:
            m.hang_np = self._p("mesh_hang_np", C.c_int8)
            m.hang_par = self._p("mesh_hang_par", C.c_int32)
        for a in range(3):
            m.lo[a], m.hi[a] = float(d["mesh_lo"][a]), float(d["mesh_hi"][a])
        m.locate_tol = float(d["mesh_locate_tol"])
        return m

    def rays_struct(self, a):
        r = N.PbgpuRays()
        pre = "rays%d_" % a
        r.n_rays = len(self.d[pre + "keys"])
        r.keys = self._p(pre + "keys", C.c_uint64)
        r.ptr = self._p(pre + "ptr", C.c_int64)
        r.inters = self._p(pre + "inters", C.c_double)
        r.normals = self._p(pre + "normals", C.c_double)
        return r

    def atoms(self):
        q = self.d["atoms_q"]
        return self.d["atoms_pos"], q, np.zeros_like(q)

    def model(self):
        md = N.PbgpuModel()
        for (k, t), v in zip(md._fields_, self.d["model"]):
            setattr(md, k, t(int(v)).value if t is C.c_int else float(v))
        return md

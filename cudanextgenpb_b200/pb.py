"""Python face of the PB path: the host problem (pbhost) and the GPU path (pbgpu).

``Problem`` mirrors the reference's set-up half of ``poisson_boltzmann``
(parse_options, read_atoms_from_pqr, create_mesh, init_tmesh*, refine_surface;
src/pb_class.cpp:39-1745) and exposes the mesh, ray and atom arrays that feed
the GPU.  ``GpuPath`` mirrors the hot half (create_markers, create_density_map,
assemple_system_matrix, lis_compute_electric_potential,
write_potential_on_atoms_fast, energy / energy_fast) one call per reference
member function, through the C ABI of include/pbgpu.h.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _native as N


class PBError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__("pbgpu status %d: %s" % (code, msg))
        self.code = code


def _arr(ptr, count, dtype):
    if count == 0:
        return np.zeros(0, dtype=dtype)
    return np.ctypeslib.as_array(ptr, shape=(count,)).astype(dtype, copy=True)


def _dptr(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


class Problem:
    """Options + atoms + octree + surface rays, built by libpbhost."""

    def __init__(self, options_text: str | None = None, options_file: str | None = None):
        self._lib = N.load_host()
        self._h = self._lib.pbhost_create()
        if not self._h:
            raise MemoryError("pbhost_create failed")
        if options_file:
            self._check(self._lib.pbhost_load_options_file(self._h, options_file.encode()))
        if options_text:
            self._check(self._lib.pbhost_load_options_text(self._h, options_text.encode()))

    def _check(self, st):
        if st != 0:
            raise PBError(st, self._lib.pbhost_last_error(self._h).decode())

    def close(self):
        if self._h:
            self._lib.pbhost_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_option(self, key: str, value):
        self._check(self._lib.pbhost_set_option(self._h, key.encode(), str(value).encode()))

    def read_pqr(self, path: str):
        self._check(self._lib.pbhost_read_pqr(self._h, path.encode()))

    def set_atoms(self, pos, charge, radius):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(charge, dtype=np.float64)
        r = np.ascontiguousarray(radius, dtype=np.float64)
        self._check(self._lib.pbhost_set_atoms(self._h, len(q), _dptr(pos), _dptr(q), _dptr(r)))

    def build(self):
        self._check(self._lib.pbhost_build_problem(self._h))
        return self

    def info(self) -> dict:
        inf = N.PbhostInfo()
        self._check(self._lib.pbhost_get_info(self._h, C.byref(inf)))
        out = {}
        for k, _ in inf._fields_:
            v = getattr(inf, k)
            out[k] = list(v) if hasattr(v, "__len__") else v
        return out

    def mesh_build(self, on_gpu: bool = True) -> N.PbgpuMeshBuild:
        """The host half of build_on_gpu alone: the pbgpu_mesh_build input of
        GpuPath.build_mesh or of a server request.  on_gpu leaves the initial
        octree (init_tmesh*) to the GPU; otherwise it is built here.  Its
        arrays belong to this problem (valid until the next call)."""
        b = N.PbgpuMeshBuild()
        self._check(self._lib.pbhost_initial_octree(self._h, 1 if on_gpu else 0, C.byref(b)))
        return b

    def build_on_gpu(self, g: "GpuPath") -> "GpuPath":
        """Domain and initial octree here, surface refinement, nodes and ray
        tables on the GPU into g's context (which also gets the atoms and the
        model); returns g, ready for create_markers."""
        self._check(self._lib.pbhost_build_on_gpu(self._h, g._ctx))
        no, nn, nh = C.c_int64(), C.c_int64(), C.c_int64()
        nr = (C.c_int64 * 3)()
        g._check(g._lib.pbgpu_get_mesh_counts(g._ctx, C.byref(no), C.byref(nn), C.byref(nh), nr))
        g.n, g.n_oct, g.n_hang = nn.value, no.value, nh.value
        g.n_rays = list(nr)
        pos, q, _ = self.atoms()
        g.n_atoms = len(q)
        return g

    def write_vtu(self, basename: str, fieldname: str, values) -> str:
        """One node field on this problem's mesh to <basename>_0000.vtu (the
        reference's VTU layout); returns the file name."""
        v = np.ascontiguousarray(values, dtype=np.float64)
        self._check(self._lib.pbhost_write_vtu(self._h, basename.encode(), fieldname.encode(), _dptr(v)))
        return "%s_0000.vtu" % basename

    def mesh_struct(self) -> N.PbgpuMesh:
        m = N.PbgpuMesh()
        self._check(self._lib.pbhost_get_mesh(self._h, C.byref(m)))
        return m

    def rays_struct(self, axis: int) -> N.PbgpuRays:
        r = N.PbgpuRays()
        self._check(self._lib.pbhost_get_rays(self._h, axis, C.byref(r)))
        return r

    def mesh(self) -> dict:
        m = self.mesh_struct()
        return {
            "n_oct": m.n_oct, "n_nodes": m.n_nodes, "n_hang": m.n_hang,
            "oct_xyz": _arr(m.oct_xyz, 3 * m.n_oct, np.int32).reshape(-1, 3),
            "oct_level": _arr(m.oct_level, m.n_oct, np.int8),
            "oct_nodes": _arr(m.oct_nodes, 8 * m.n_oct, np.int32).reshape(-1, 8),
            "node_xyz": _arr(m.node_xyz, 3 * m.n_nodes, np.int32).reshape(-1, 3),
            "hang_np": _arr(m.hang_np, m.n_hang, np.int8),
            "hang_par": _arr(m.hang_par, 4 * m.n_hang, np.int32).reshape(-1, 4),
            "lo": np.array(list(m.lo)), "hi": np.array(list(m.hi)), "locate_tol": m.locate_tol,
        }

    def rays(self, axis: int) -> dict:
        r = self.rays_struct(axis)
        ptr = _arr(r.ptr, r.n_rays + 1, np.int64)
        nc = int(ptr[-1]) if r.n_rays else 0
        return {"keys": _arr(r.keys, r.n_rays, np.uint64), "ptr": ptr, "inters": _arr(r.inters, nc, np.float64),
                "normals": _arr(r.normals, 3 * nc, np.float64).reshape(-1, 3)}

    def atoms(self):
        n = self.info()["n_atoms"]
        pos = np.zeros((n, 3))
        q = np.zeros(n)
        r = np.zeros(n)
        self._check(self._lib.pbhost_get_atoms(self._h, _dptr(pos), _dptr(q), _dptr(r)))
        return pos, q, r

    def model(self) -> N.PbgpuModel:
        m = N.PbgpuModel()
        self._check(self._lib.pbhost_get_model(self._h, C.byref(m)))
        return m

    def solver_opts(self) -> N.PbgpuSolverOpts:
        o = N.PbgpuSolverOpts()
        self._check(self._lib.pbhost_get_solver_opts(self._h, C.byref(o)))
        return o

    def run_gpu(self):
        """The whole path through the host mirror's run_gpu_path (the driver order)."""
        e, s = N.PbgpuEnergyOut(), N.PbgpuSolveStats()
        st = self._lib.pbhost_run_gpu(self._h, C.byref(e), C.byref(s))
        if st not in (0, N.PBGPU_NOT_CONVERGED):
            raise PBError(st, self._lib.pbhost_last_error(self._h).decode())
        return e.as_dict(), s


def solver_opts(method="cg", tol=1e-8, max_iter=20000, precision="fp64", inner_tol=1e-5, check_every=16,
                max_outer=50, precond="jacobi", conv_cond=0, tol_w=1.0) -> N.PbgpuSolverOpts:
    o = N.PbgpuSolverOpts()
    N.load_gpu().pbgpu_default_solver_opts(C.byref(o))
    o.method = {"cg": N.PBGPU_CG, "bicgstab": N.PBGPU_BICGSTAB, "cgs": N.PBGPU_CGS}[method]
    o.precond = {"none": N.PBGPU_PRECOND_NONE, "jacobi": N.PBGPU_PRECOND_JACOBI,
                 "block_jacobi": N.PBGPU_PRECOND_BLOCK_JACOBI}[precond]
    o.precision = {"fp64": N.PBGPU_FP64, "mixed": N.PBGPU_MIXED}[precision]
    o.tol, o.max_iter, o.inner_tol, o.check_every, o.max_outer = tol, max_iter, inner_tol, check_every, max_outer
    o.conv_cond, o.tol_w = conv_cond, tol_w
    return o


def parse_lis_options(text: str) -> N.PbgpuSolverOpts:
    o = N.PbgpuSolverOpts()
    st = N.load_gpu().pbgpu_parse_lis_options(text.encode(), C.byref(o))
    if st != 0:
        raise PBError(st, "bad LIS option string: %r" % text)
    return o


class GpuPath:
    """One pbgpu context: the reference's hot-path member functions on the GPU."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self._lib = N.load_gpu()
        self._ctx = C.c_void_p()
        st = self._lib.pbgpu_ctx_create(C.byref(self._ctx), device, C.c_void_p(stream) if stream else None)
        if st != 0:
            raise PBError(st, "pbgpu_ctx_create failed (no CUDA device?)")
        self.n = self.n_oct = self.n_atoms = 0

    def _check(self, st, ok=(0,)):
        if st not in ok:
            raise PBError(st, self._lib.pbgpu_last_error(self._ctx).decode())
        return st

    def close(self):
        if self._ctx:
            self._lib.pbgpu_ctx_destroy(self._ctx)
            self._ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # ---- inputs
    def load(self, prob: Problem):
        m = prob.mesh_struct()
        self._check(self._lib.pbgpu_set_mesh(self._ctx, C.byref(m)))
        for a in range(3):
            r = prob.rays_struct(a)
            self._check(self._lib.pbgpu_set_rays(self._ctx, a, C.byref(r)))
        pos, q, _ = prob.atoms()
        self.set_atoms(pos, q)
        md = prob.model()
        self._check(self._lib.pbgpu_set_model(self._ctx, C.byref(md)))
        self.n, self.n_oct = m.n_nodes, m.n_oct
        return self

    def build_mesh(self, build: N.PbgpuMeshBuild):
        """pbgpu_build_mesh: surface refinement, nodes and ray tables on the GPU
        from a host initial octree (Problem.mesh_build())."""
        self._check(self._lib.pbgpu_build_mesh(self._ctx, C.byref(build)))
        no, nn, nh = C.c_int64(), C.c_int64(), C.c_int64()
        nr = (C.c_int64 * 3)()
        self._check(self._lib.pbgpu_get_mesh_counts(self._ctx, C.byref(no), C.byref(nn), C.byref(nh), nr))
        self.n, self.n_oct, self.n_hang = nn.value, no.value, nh.value
        self.n_rays = list(nr)
        return self

    def set_atoms(self, pos, q):
        pos = np.ascontiguousarray(pos, dtype=np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(q, dtype=np.float64)
        self._check(self._lib.pbgpu_set_atoms(self._ctx, len(q), _dptr(pos), _dptr(q)))
        self.n_atoms = len(q)

    def set_model(self, model: N.PbgpuModel):
        self._check(self._lib.pbgpu_set_model(self._ctx, C.byref(model)))

    # ---- path
    def create_markers(self):
        self._check(self._lib.pbgpu_create_markers(self._ctx))

    def create_density_map(self):
        self._check(self._lib.pbgpu_create_density_map(self._ctx))

    def assemble(self, chunk=32, sigma=2048, group=4):
        """SELL-C-sigma layout: slice height `chunk`, length-sorting window
        `sigma` rows, `group` columns stored contiguously per row."""
        o = N.PbgpuSellOpts(chunk, sigma, group)
        self._check(self._lib.pbgpu_assemble(self._ctx, C.byref(o)))

    def autotune(self, iterations: int = 24) -> dict:
        """Time the SpMV in each candidate SELL layout; the fastest stays assembled."""
        so, cols, ms = N.PbgpuSellOpts(), C.c_int(), C.c_double()
        self._check(self._lib.pbgpu_autotune(self._ctx, iterations, C.byref(so), C.byref(cols), C.byref(ms)))
        return {"chunk": so.chunk, "sigma": so.sigma, "group": so.group, "cols": cols.value, "spmv_ms": ms.value}

    def solve(self, opts: N.PbgpuSolverOpts | None = None, allow_not_converged=False):
        s = N.PbgpuSolveStats()
        ok = (0, N.PBGPU_NOT_CONVERGED) if allow_not_converged else (0,)
        self._check(self._lib.pbgpu_solve(self._ctx, C.byref(opts) if opts else None, C.byref(s)), ok)
        return s

    def phi_on_atoms(self):
        out = np.zeros(self.n_atoms)
        self._check(self._lib.pbgpu_phi_on_atoms(self._ctx, _dptr(out)))
        return out

    def energy(self, fast=False) -> dict:
        e = N.PbgpuEnergyOut()
        self._check(self._lib.pbgpu_energy(self._ctx, 1 if fast else 0, C.byref(e)))
        return e.as_dict()

    def pot_field(self, calc_potential_terms: int, calc_field_terms: int, fast=False):
        """pot_field / pot_field_fast: (per-atom rows of the 12 columns in
        N.POT_FIELD_COLUMNS order, dict of energies and the `columns` bitmask
        of those the reference writes)."""
        rows = np.zeros((self.n_atoms, len(N.POT_FIELD_COLUMNS)))
        o = N.PbgpuPotFieldOut()
        self._check(self._lib.pbgpu_pot_field(self._ctx, 1 if fast else 0, int(calc_potential_terms),
                                              int(calc_field_terms), _dptr(rows), C.byref(o)))
        return rows, o.as_dict()

    # ---- read-back
    def mesh_arrays(self) -> dict:
        """The context's mesh (set or built on the GPU) as numpy arrays in the
        layout of Problem.mesh()."""
        no, nn, nh = C.c_int64(), C.c_int64(), C.c_int64()
        nr = (C.c_int64 * 3)()
        self._check(self._lib.pbgpu_get_mesh_counts(self._ctx, C.byref(no), C.byref(nn), C.byref(nh), nr))
        no, nn, nh = no.value, nn.value, nh.value
        d = {"oct_xyz": np.zeros((no, 3), np.int32), "oct_level": np.zeros(no, np.int8),
             "oct_nodes": np.zeros((no, 8), np.int32), "node_xyz": np.zeros((nn, 3), np.int32),
             "hang_np": np.zeros(nh, np.int8), "hang_par": np.zeros((nh, 4), np.int32)}
        box = np.zeros(6)
        P = C.POINTER
        i32 = lambda a: a.ctypes.data_as(P(C.c_int32))
        i8 = lambda a: a.ctypes.data_as(P(C.c_int8))
        self._check(self._lib.pbgpu_get_mesh(self._ctx, i32(d["oct_xyz"]), i8(d["oct_level"]), i32(d["oct_nodes"]),
                                             i32(d["node_xyz"]), i8(d["hang_np"]), i32(d["hang_par"]), _dptr(box)))
        d["lo"], d["extent"] = box[:3].copy(), box[3:].copy()
        return d

    def node_coeffs(self):
        eps, react = np.zeros(self.n), np.zeros(self.n)
        self._check(self._lib.pbgpu_get_node_coeffs(self._ctx, _dptr(eps), _dptr(react)))
        return eps, react

    def markers(self):
        marker = np.zeros(self.n_oct)
        nb = C.c_int64()
        self._check(self._lib.pbgpu_get_markers(self._ctx, _dptr(marker), C.byref(nb), None))
        border = np.zeros(nb.value, dtype=np.int32)
        self._check(self._lib.pbgpu_get_markers(self._ctx, None, C.byref(nb),
                                                border.ctypes.data_as(C.POINTER(C.c_int32))))
        return marker, border

    def fractions(self, n_border):
        f = np.zeros(12 * n_border)
        self._check(self._lib.pbgpu_get_fractions(self._ctx, _dptr(f)))
        return f.reshape(-1, 12)

    def density(self):
        rho, vp = np.zeros(self.n), np.zeros(self.n)
        self._check(self._lib.pbgpu_get_density(self._ctx, _dptr(rho), _dptr(vp)))
        return rho, vp

    def system(self):
        nnz = C.c_int64()
        self._check(self._lib.pbgpu_get_system(self._ctx, C.byref(nnz), None, None, None, None))
        rp = np.zeros(self.n + 1, dtype=np.int64)
        col = np.zeros(nnz.value, dtype=np.int32)
        val = np.zeros(nnz.value)
        rhs = np.zeros(self.n)
        self._check(self._lib.pbgpu_get_system(self._ctx, C.byref(nnz), rp.ctypes.data_as(C.POINTER(C.c_int64)),
                                               col.ctypes.data_as(C.POINTER(C.c_int32)), _dptr(val), _dptr(rhs)))
        return rp, col, val, rhs

    def phi(self):
        out = np.zeros(self.n)
        self._check(self._lib.pbgpu_get_phi(self._ctx, _dptr(out)))
        return out

    def stage_ms(self):
        ms = (C.c_double * 6)()
        self._check(self._lib.pbgpu_get_stage_ms(self._ctx, ms))
        return dict(zip(["markers", "density", "assemble", "solve", "phi_atoms", "energy"], list(ms)))

    def stream_ptr(self) -> int:
        """cudaStream_t of this context (e.g. for torch.cuda.ExternalStream)."""
        return int(self._lib.pbgpu_ctx_stream(self._ctx) or 0)

    def set_profiling(self, on=True):
        self._check(self._lib.pbgpu_set_profiling(self._ctx, 1 if on else 0))

    def set_wait_limit(self, seconds: float):
        """Limit of each bounded device-side wait of this context (0: give up at once)."""
        self._check(self._lib.pbgpu_set_wait_limit(self._ctx, float(seconds)))

    def counters(self) -> dict:
        c = N.PbgpuCounters()
        self._check(self._lib.pbgpu_get_counters(self._ctx, C.byref(c)))
        return {k: getattr(c, k) for k, _ in c._fields_}

    def reset_counters(self):
        self._check(self._lib.pbgpu_reset_counters(self._ctx))

    def run(self, opts=None, fast=False, chunk=32, sigma=2048, group=4):
        """create_markers .. energy in the driver's order; returns (energy dict, solve stats)."""
        self.create_markers()
        self.create_density_map()
        self.assemble(chunk, sigma, group)
        st = self.solve(opts)
        return self.energy(fast), st


class Batch:
    """Many assembled GpuPath systems solved together by one persistent
    cooperative kernel per chunk of iterations (pbgpu_batch_*)."""

    def __init__(self, device: int = 0, stream: int | None = None):
        self._lib = N.load_gpu()
        self._b = C.c_void_p()
        st = self._lib.pbgpu_batch_create(C.byref(self._b), device, C.c_void_p(stream) if stream else None)
        if st != 0:
            raise PBError(st, "pbgpu_batch_create failed")
        self.members: dict[int, GpuPath] = {}

    def _check(self, st, ok=(0,)):
        if st not in ok:
            raise PBError(st, self._lib.pbgpu_batch_last_error(self._b).decode())

    def add(self, g: GpuPath) -> int:
        slot = C.c_int()
        self._check(self._lib.pbgpu_batch_add(self._b, g._ctx, C.byref(slot)))
        self.members[slot.value] = g
        return slot.value

    def remove(self, slot: int):
        self._check(self._lib.pbgpu_batch_remove(self._b, slot))
        del self.members[slot]

    def solve(self, opts: N.PbgpuSolverOpts | None = None, allow_not_converged=False) -> dict:
        n = max(self.members) + 1 if self.members else 0
        stats = (N.PbgpuSolveStats * max(n, 1))()
        ok = (0, N.PBGPU_NOT_CONVERGED) if allow_not_converged else (0,)
        self._check(self._lib.pbgpu_batch_solve(self._b, C.byref(opts) if opts else None, stats), ok)
        return {k: stats[k] for k in self.members}

    def begin(self, opts: N.PbgpuSolverOpts | None = None):
        self._check(self._lib.pbgpu_batch_begin(self._b, C.byref(opts) if opts else None))

    def step(self, steps: int) -> int:
        """One persistent launch of up to `steps` steps; returns the members not done."""
        n = C.c_int()
        self._check(self._lib.pbgpu_batch_step(self._b, steps, C.byref(n)))
        return n.value

    def member(self, slot: int):
        """(done, stats) of a member; when done its potential is in its context."""
        done, st = C.c_int(), N.PbgpuSolveStats()
        self._check(self._lib.pbgpu_batch_member(self._b, slot, C.byref(done), C.byref(st)))
        return bool(done.value), st

    def set_blocks_per_sm(self, blocks: int):
        self._check(self._lib.pbgpu_batch_set_blocks_per_sm(self._b, blocks))

    def set_wait_limit(self, seconds: float):
        """Limit of each member-barrier wait in the persistent kernel (0: give up at once)."""
        self._check(self._lib.pbgpu_batch_set_wait_limit(self._b, float(seconds)))

    def close(self):
        if self._b:
            self._lib.pbgpu_batch_destroy(self._b)
            self._b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class Server:
    """Continuous-batching PB solve server on one GPU (pbgpu_server_*).

    submit(problem) queues one molecule (its host arrays stay referenced until
    its result comes back); progress() runs one tick and returns finished
    requests as dicts."""

    def __init__(self, device: int = 0, opts: N.PbgpuServerOpts | None = None, **kw):
        self._lib = N.load_gpu()
        if opts is None:
            opts = N.PbgpuServerOpts()
            self._lib.pbgpu_default_server_opts(C.byref(opts))
        for k, v in kw.items():
            if k in ("tol", "inner_tol", "max_iter", "precision", "check_every"):
                if k == "precision":
                    v = {"fp64": N.PBGPU_FP64, "mixed": N.PBGPU_MIXED}[v]
                setattr(opts.solver, k, v)
            else:
                setattr(opts, k, v)
        self.opts = opts
        self._s = C.c_void_p()
        st = self._lib.pbgpu_server_create(C.byref(self._s), device, C.byref(opts))
        if st != 0:
            raise PBError(st, "pbgpu_server_create failed")
        self._keep: dict[int, tuple] = {}
        self._out = (N.PbgpuResult * 256)()

    def _check(self, st):
        if st != 0:
            raise PBError(st, self._lib.pbgpu_server_last_error(self._s).decode())

    def request(self, prob: Problem, pos=None, q=None, tag: int = 0, build: N.PbgpuMeshBuild | None = None
                ) -> N.PbgpuRequest:
        """The request structure of a built host problem (optionally with other
        charges on the same atoms), or, with `build` (Problem.mesh_build()), of
        a problem whose mesh the server builds on the GPU."""
        p0, q0, _ = prob.atoms()
        pos = np.ascontiguousarray(p0 if pos is None else pos, dtype=np.float64).reshape(-1, 3)
        q = np.ascontiguousarray(q0 if q is None else q, dtype=np.float64)
        md = prob.model()
        r = N.PbgpuRequest()
        m = None
        if build is not None:
            r.build = C.pointer(build)
        else:
            m = prob.mesh_struct()
            r.mesh = C.pointer(m)
            for a in range(3):
                r.rays[a] = prob.rays_struct(a)
        r.n_atoms = len(q)
        r.pos = _dptr(pos)
        r.charge = _dptr(q)
        r.model = C.pointer(md)
        r.user_tag = tag
        r._keep = (m, pos, q, md, prob, build)
        return r

    def submit(self, req: N.PbgpuRequest) -> int:
        i = C.c_int64()
        self._check(self._lib.pbgpu_server_submit(self._s, C.byref(req), C.byref(i)))
        self._keep[i.value] = (req, req._keep)
        return i.value

    def progress(self) -> list[dict]:
        n = C.c_int()
        self._check(self._lib.pbgpu_server_progress(self._s, self._out, len(self._out), C.byref(n)))
        res = []
        for k in range(n.value):
            r = self._out[k]
            self._keep.pop(r.id, None)
            res.append({"id": r.id, "tag": r.user_tag, "status": r.status, "energy": r.energy.as_dict(),
                        "iterations": r.stats.iterations, "outer": r.stats.outer,
                        "rel_residual": r.stats.rel_residual, "latency_ms": r.latency_ms, "queue_ms": r.queue_ms})
        return res

    def pending(self):
        q, r, b = C.c_int(), C.c_int(), C.c_int64()
        self._check(self._lib.pbgpu_server_pending(self._s, C.byref(q), C.byref(r), C.byref(b)))
        return q.value, r.value, b.value

    def stats(self) -> dict:
        """Requests admitted / completed / rejected and kernels launched so far."""
        a, c, r, l = C.c_int64(), C.c_int64(), C.c_int64(), C.c_int64()
        self._check(self._lib.pbgpu_server_stats(self._s, C.byref(a), C.byref(c), C.byref(r), C.byref(l)))
        return {"admitted": a.value, "completed": c.value, "rejected": r.value, "launches": l.value}

    def estimate(self, req: N.PbgpuRequest) -> int:
        return int(self._lib.pbgpu_request_bytes_estimate(C.byref(req)))

    def close(self):
        if self._s:
            self._lib.pbgpu_server_destroy(self._s)
            self._s = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def solve_charges(g: GpuPath, charges, opts: N.PbgpuSolverOpts | None = None, fast=False):
    """k charge vectors (k x n_atoms) on g's assembled system in one multi-RHS
    solve; returns (list of energy dicts, list of solve stats)."""
    q = np.ascontiguousarray(charges, dtype=np.float64)
    k = q.shape[0]
    es = (N.PbgpuEnergyOut * k)()
    ss = (N.PbgpuSolveStats * k)()
    g._check(g._lib.pbgpu_solve_charges(g._ctx, k, _dptr(q), C.byref(opts) if opts else None, 1 if fast else 0,
                                        es, ss))
    return [e.as_dict() for e in es], list(ss)

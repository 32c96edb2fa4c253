"""Benchmark of the PB path (one JSON line on rank 0).

Default workload (`serve`): a seeded stream of PB requests, each a synthetic
molecule (atoms log-uniform in 200-2,000, scale 2/A, 1 or 2 surface levels).
A request is served whole on the GPU: the mesh (initial octree, surface
refinement, nodes, hanging nodes, ray tables), create_markers,
create_density_map, assembly (SELL-C-sigma), the Krylov solve and the energy.
The same requests run twice in one process:

  served  the continuous-batching server, worker contexts each serving whole
          requests on their own stream, FP32-inner / FP64-refined CG;
  plain   one request at a time through the plain FP64 path.

value            served solves/s (all timed requests offered at once);
latency_ms       p50/p95/p99 from arrival to result under Poisson arrivals at
                 70 % of that capacity;
speedup_vs_plain_fp64, and the energy error of every served request against
the plain FP64 result and, on three molecules, against the CPU oracle.
roofline         the CG SpMV of the plain FP64 path on the 2,000-atom molecule.

Single-molecule workloads (`mol2000`, `mol2000l2`, `mol25k`, ...) time one
molecule's whole path per step (value: inputs resident in HBM; e2e: through
the C ABI from pinned host buffers).  Multi-GPU (torchrun, or --gpus N which
starts it): replicas, one process per GPU, timing the max over ranks.
--impl reference times the CPU oracle, whole solves, with inputs prepared in a
separate process.
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

METRIC = "PB solves/s + p50/p99 latency vs plain FP64 GPU solve at <=1e-6 energy err"
FALLBACK_HBM_GBS = 6650.0

WORKLOADS = {
    # name: (n_atoms, radius, net charge, seed, scale, levels)
    "mol2000": (2000, 18.0, -3.0, 2000, 2.0, 3),
    # same molecule, 2 surface levels: the profiling case (inputs > L2, ~2 GB on device)
    "mol2000l2": (2000, 18.0, -3.0, 2000, 2.0, 2),
    "mol300": (300, 11.0, -3.0, 300, 2.0, 2),
    "mol60": (60, 7.0, -3.0, 60, 2.0, 1),
    # the 25,000-atom complex (radius 45 A, net +7 e, seed 25000) at scale 2/A
    # with 2 surface levels: the mixed-precision configuration, scaled so the
    # host mesh build stays within a minute
    "mol25k": (25000, 45.0, 7.0, 25000, 2.0, 2),
}


def log(*a):
    print(*a, file=sys.stderr, flush=True)


def max_over_ranks(value, dist, device="cuda"):
    """The largest of the ranks' values: a multi-GPU step takes as long as its
    slowest rank."""
    if not dist:
        return value
    import torch
    t = torch.tensor([float(value)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def replicas_throughput(world, steps, ms_max):
    """Whole-job solves/s of `world` independent replicas that each ran
    `steps` solves, timed by the slowest rank."""
    return world * steps / (ms_max / 1e3)


def dist_env():
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", str(rank)))
    return rank, world, local


class Clocks:
    """nvidia-smi samples of SM clock and throttle reasons during the timed region."""

    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, gpu_index):
        self.idx = gpu_index
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.idx), "--query-gpu=" + self.Q,
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def stop(self):
        if not self.proc:
            return None
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in self.lines:
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx.append(float(f[2]))
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": float(max(mx)), "reasons": sorted(reasons),
                "samples": len(sm)}


def measured_peak():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        d = json.load(open(p))
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return FALLBACK_HBM_GBS, "fallback"


def spmv_traffic():
    """DRAM bytes per SpMV launch of each kernel from the committed ncu
    summaries (captured on a smaller case; scaled to the bench workload by nnz)."""
    p = os.path.join(ROOT, "profiles", "spmv_traffic.json")
    try:
        return json.load(open(p))
    except Exception:
        return None


def spmv_kernel_name(args):
    """The CG SpMV kernel the solve runs for the bench's layout."""
    if args.chunk == 32 and args.group == 1 and os.environ.get("PBGPU_SPMV") != "direct":
        return "k_cg_spmv_tma<double, %s>" % os.environ.get("PBGPU_SPMV_COLS", "16")
    if args.group == 4 and os.environ.get("PBGPU_SPMV_PAIRS", "1") != "0":
        return "k_cg_spmv<double, 8>"  # the G = 4 layout walked two column groups per iteration
    return "k_cg_spmv<double, %d>" % args.group


def build_problem(name):
    from cudanextgenpb_b200 import configs
    na, rad, net, seed, scale, levels = WORKLOADS[name]
    prob = configs.make_globular_problem(na, rad, net, seed, scale=scale, levels=levels)
    t0 = time.time()
    prob.build()
    prob.host_build_s = time.time() - t0
    log("host problem %s built in %.1fs: %s" % (name, prob.host_build_s,
                                                 {k: prob.info()[k] for k in ("n_oct", "n_nodes", "n_hang")}))
    return prob


def gpu_mesh_build_s(name, device, repeats=2):
    """Seconds of the same problem's set-up with the surface refinement, nodes
    and ray tables built on the GPU (Problem.build_on_gpu): first call, and the
    best of the repeats after it."""
    from cudanextgenpb_b200 import GpuPath, configs
    na, rad, net, seed, scale, levels = WORKLOADS[name]
    times = []
    for _ in range(1 + repeats):
        p = configs.make_globular_problem(na, rad, net, seed, scale=scale, levels=levels)
        g = GpuPath(device)
        t0 = time.time()
        p.build_on_gpu(g)
        times.append(time.time() - t0)
        g.close()
    return times[0], min(times[1:])


def pinned_inputs(prob):
    """Copies of the mesh / ray / atom host arrays in pinned memory, and the
    pbgpu structures pointing at them."""
    import ctypes as C

    import torch

    from cudanextgenpb_b200 import _native as N
    keep = []

    def pin(a):
        t = torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
        keep.append(t)
        return t

    def ptr(t, ct):
        return C.cast(C.c_void_p(t.data_ptr()), C.POINTER(ct))

    m = prob.mesh()
    ms = N.PbgpuMesh()
    ms.n_oct, ms.n_nodes, ms.n_hang = m["n_oct"], m["n_nodes"], m["n_hang"]
    t = pin(m["oct_xyz"].reshape(-1)); ms.oct_xyz = ptr(t, C.c_int32)
    t = pin(m["oct_level"]); ms.oct_level = ptr(t, C.c_int8)
    t = pin(m["oct_nodes"].reshape(-1)); ms.oct_nodes = ptr(t, C.c_int32)
    t = pin(m["node_xyz"].reshape(-1)); ms.node_xyz = ptr(t, C.c_int32)
    t = pin(m["hang_np"] if m["n_hang"] else np.zeros(1, np.int8)); ms.hang_np = ptr(t, C.c_int8)
    t = pin(m["hang_par"].reshape(-1) if m["n_hang"] else np.zeros(4, np.int32)); ms.hang_par = ptr(t, C.c_int32)
    for a in range(3):
        ms.lo[a], ms.hi[a] = m["lo"][a], m["hi"][a]
    ms.locate_tol = m["locate_tol"]
    h2d = sum(int(x.numel() * x.element_size()) for x in keep)
    rays = []
    for a in range(3):
        r = prob.rays(a)
        rs = N.PbgpuRays()
        rs.n_rays = len(r["keys"])
        k0 = len(keep)
        t = pin(r["keys"].view(np.int64)); rs.keys = ptr(t, C.c_uint64)
        t = pin(r["ptr"]); rs.ptr = ptr(t, C.c_int64)
        t = pin(r["inters"]); rs.inters = ptr(t, C.c_double)
        t = pin(r["normals"].reshape(-1)); rs.normals = ptr(t, C.c_double)
        h2d += sum(int(x.numel() * x.element_size()) for x in keep[k0:])
        rays.append(rs)
    pos, q, _ = prob.atoms()
    tp, tq = pin(pos.reshape(-1)), pin(q)
    h2d += int(tp.numel() * 8 + tq.numel() * 8)
    return {"mesh": ms, "rays": rays, "pos": ptr(tp, C.c_double), "q": ptr(tq, C.c_double), "na": len(q),
            "model": prob.model(), "keep": keep, "h2d_bytes": h2d}


def run_ours(args, rank, world, local):
    import ctypes as C

    import torch

    from cudanextgenpb_b200 import GpuPath, solver_opts
    from cudanextgenpb_b200 import _native as N

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))

    prob = build_problem(args.workload)
    g = GpuPath(local).load(prob)
    # time on the context's own stream
    stream = torch.cuda.ExternalStream(g.stream_ptr(), device=local)
    opts = solver_opts("cg", tol=args.tol, max_iter=50000, precond=args.precond, precision=args.precision)
    info = prob.info()

    batch = None
    if args.via_batch:
        from cudanextgenpb_b200 import Batch
        batch = Batch(local)
        opts = solver_opts("cg", tol=args.tol, max_iter=50000, precision=args.precision, check_every=64)

    def step():
        g.create_markers()
        g.create_density_map()
        g.assemble(args.chunk, args.sigma, args.group)
        if batch is not None:
            batch.add(g)
            st = batch.solve(opts)[0]
            batch.remove(0)
        else:
            st = g.solve(opts)
        pa = g.phi_on_atoms()
        e = g.energy(False)
        return st, e, pa

    # warm-up
    for _ in range(args.warmup):
        st, e, _ = step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    # the timed steps run without per-SpMV events (value and e2e alike); the
    # SpMV roofline comes from a separate profiled pass after them
    g.reset_counters()
    clocks = Clocks(local)
    clocks.start()
    t_start = torch.cuda.Event(enable_timing=True)
    t_end = torch.cuda.Event(enable_timing=True)
    lat = []
    energies = []
    iters = []
    t_start.record(stream)
    for _ in range(args.steps):
        a = torch.cuda.Event(enable_timing=True)
        b = torch.cuda.Event(enable_timing=True)
        a.record(stream)
        st, e, _ = step()
        b.record(stream)
        b.synchronize()
        lat.append(a.elapsed_time(b))
        energies.append(e["sum"])
        iters.append(st.iterations)
    t_end.record(stream)
    torch.cuda.synchronize()
    ck = clocks.stop()
    ms = t_start.elapsed_time(t_end)
    cnt = g.counters()
    stage = g.stage_ms()
    # SpMV launch times: CUDA events around every SpMV of two more solves
    g.set_profiling(True)
    c0 = g.counters()
    for _ in range(2):
        g.solve(opts)
    c1 = g.counters()
    g.set_profiling(False)
    cnt = dict(cnt, spmv_ms=c1["spmv_ms"] - c0["spmv_ms"], spmv_launches=c1["spmv_launches"] - c0["spmv_launches"],
               spmv_bytes=c1["spmv_bytes"])
    ms = max_over_ranks(ms, dist)
    if dist:
        dist.barrier()

    # end to end through the C ABI from pinned host buffers
    lib = N.load_gpu()
    pin = pinned_inputs(prob)
    ctx = g._ctx
    out_atoms = torch.empty(pin["na"], dtype=torch.float64).pin_memory()
    e_out = N.PbgpuEnergyOut()

    def e2e_step():
        assert lib.pbgpu_set_mesh(ctx, C.byref(pin["mesh"])) == 0
        for a in range(3):
            assert lib.pbgpu_set_rays(ctx, a, C.byref(pin["rays"][a])) == 0
        assert lib.pbgpu_set_atoms(ctx, pin["na"], pin["pos"], pin["q"]) == 0
        assert lib.pbgpu_set_model(ctx, C.byref(pin["model"])) == 0
        assert lib.pbgpu_create_markers(ctx) == 0
        assert lib.pbgpu_create_density_map(ctx) == 0
        so = N.PbgpuSellOpts(args.chunk, args.sigma, args.group)
        assert lib.pbgpu_assemble(ctx, C.byref(so)) == 0
        s = N.PbgpuSolveStats()
        assert lib.pbgpu_solve(ctx, C.byref(opts), C.byref(s)) == 0
        assert lib.pbgpu_phi_on_atoms(ctx, C.cast(C.c_void_p(out_atoms.data_ptr()), C.POINTER(C.c_double))) == 0
        assert lib.pbgpu_energy(ctx, 0, C.byref(e_out)) == 0

    e2e_step()
    if dist:
        dist.barrier()
    torch.cuda.synchronize()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    for _ in range(args.steps):
        e2e_step()
    e1.record(stream)
    torch.cuda.synchronize()
    ms_e2e = max_over_ranks(e0.elapsed_time(e1), dist)

    # pot_field (the refined-mesh variant) on the solved system, outside the
    # timed region: per-atom Coulomb, polarisation and ionic potentials and
    # fields (calc_potential_terms = calc_field_terms = 2); the time of a call
    # includes its host synchronisations
    g.pot_field(2, 2)
    torch.cuda.synchronize()
    c0 = g.counters()["energy_pairs"]
    p0 = torch.cuda.Event(enable_timing=True)
    p1 = torch.cuda.Event(enable_timing=True)
    p0.record(stream)
    for _ in range(3):
        g.pot_field(2, 2)
    p1.record(stream)
    torch.cuda.synchronize()
    pf_ms = p0.elapsed_time(p1) / 3
    pf_pairs = (g.counters()["energy_pairs"] - c0) / 3
    pot_field = {"ms_per_call": pf_ms, "surface_points": g.counters()["energy_points"],
                 "atoms": info["n_atoms"], "point_atom_pairs": pf_pairs,
                 "gpairs_per_s": pf_pairs / (pf_ms / 1e3) / 1e9}
    # set-up of the same molecule with the mesh built on the GPU, against the
    # host build this run started with (outside the timed region)
    gb_first, gb_best = gpu_mesh_build_s(args.workload, local)
    mesh_build = {"host_s": prob.host_build_s, "gpu_s": gb_best, "gpu_first_call_s": gb_first,
                  "what": "domain, octree, surface refinement, nodes, hanging nodes, ray tables"}

    result = None
    if rank == 0:
        value = replicas_throughput(world, args.steps, ms)
        e2e = replicas_throughput(world, args.steps, ms_e2e)
        peak, peak_kind = measured_peak()
        spmv_avg_ms = cnt["spmv_ms"] / max(cnt["spmv_launches"], 1)
        achieved = cnt["spmv_bytes"] / (spmv_avg_ms / 1e3) / 1e9 if cnt["spmv_launches"] else None
        kname = spmv_kernel_name(args)
        tr = spmv_traffic()
        traffic = None
        if tr and kname in tr.get("kernels", {}):
            traffic = tr["kernels"][kname]["dram_bytes_per_launch"] * (info_nnz(g) / tr["nnz"])
        result = {
            "metric": METRIC,
            "value": value,
            "unit": "solves/s",
            "n_gpus": world,
            "steps": args.steps,
            "warmup": args.warmup,
            "ms_per_step": ms / args.steps,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
            "higher_is_better": True,
            "scaling": "weak",
            "vs_baseline": None,
            "dtype": "f64" if args.precision == "fp64" else "f32-inner/f64",
            "data": "synthetic",
            "config": {
                "workload": workload_desc(args.workload, info),
                "n_dof": info["n_nodes"], "n_octants": info["n_oct"], "n_hanging": info["n_hang"],
                "n_atoms": info["n_atoms"], "nnz": info_nnz(g), "cg_iterations": int(np.median(iters)),
                "tol": args.tol, "precond": args.precond, "precision": args.precision,
                "solver_path": "persistent multi-system kernel" if args.via_batch else "captured CUDA graph of kernels",
                "sell": {"C": args.chunk, "sigma": args.sigma, "group": args.group},
                "energy_kT": energies[-1],
                "dof_iterations_per_s": world * info["n_nodes"] * float(np.median(iters)) / (ms / 1e3 / args.steps),
                "stage_ms": stage,
                "energy_pairs": {
                    "points": cnt["energy_points"], "pairs_per_step": cnt["energy_pairs"] / max(args.steps, 1),
                    # 12 FP64 flops per surface-point x atom pair (dx, dy, dz, r^2, 1/r, q/r, the
                    # normal term), the count the roofline of the pair kernel uses
                    "gflops": 12.0 * cnt["energy_pairs"] / max(args.steps, 1) / (stage["energy"] / 1e3) / 1e9
                    if stage.get("energy") else None,
                },
                "pot_field": pot_field,
                "mesh_build": mesh_build,
                "l2": "inputs larger than L2 (126 MB): every step streams the mesh, matrix and vectors from HBM",
                "parallelism": "replicas (one independent solve per GPU)",
            },
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": pin["h2d_bytes"],
                    "d2h_bytes_per_step": int(8 * pin["na"] + 48)},
            "roofline": {"kernel": kname + " (SELL-C-sigma SpMV fused with p.Ap)", "bound": "hbm",
                         "achieved": achieved, "peak": peak, "unit": "GB/s",
                         "frac": (achieved / peak) if achieved else None, "peak_kind": peak_kind,
                         "traffic": traffic, "algorithmic_bytes_per_launch": cnt["spmv_bytes"],
                         "avg_launch_ms": spmv_avg_ms, "launches_timed": cnt["spmv_launches"]},
            "gpu_launches": cnt["launches"],
            "clocks": ck,
        }
        if args.compare_fp64 and args.precision == "mixed":
            # the same molecule solved in plain FP64 on the GPU: error of the
            # mixed-precision potential and energy against it, and the bytes
            # each CG iteration moves in either precision
            phi_m = g.phi().copy()
            e_m = energies[-1]
            st64 = g.solve(solver_opts("cg", tol=args.tol, max_iter=50000))
            phi_64 = g.phi()
            e_64 = g.energy(False)["sum"]
            nnz = info_nnz(g)
            n = info["n_nodes"]
            result["config"]["vs_fp64"] = {
                "phi_rel_l2_err": float(np.linalg.norm(phi_m - phi_64) / np.linalg.norm(phi_64)),
                "energy_rel_err": abs(e_m - e_64) / abs(e_64),
                "fp64_cg_iterations": st64.iterations,
                "bytes_per_iteration_fp64": 12 * nnz + 104 * n,
                "bytes_per_iteration_fp32_inner": 8 * nnz + 52 * n,
            }
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = cpu_baseline(prob, args)
    g.close()
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


def info_nnz(g):
    import ctypes as C
    nnz = C.c_int64()
    g._lib.pbgpu_get_system(g._ctx, C.byref(nnz), None, None, None, None)
    return int(nnz.value)


def workload_desc(name, info):
    na, rad, net, seed, scale, levels = WORKLOADS[name]
    return ("synthetic globular molecule: %d atoms (FCC-lattice subset in a %.0f A sphere, net %+g e, seed %d), "
            "mesh_shape 0 scale %g/A, %d surface levels -> %d DoF; FP64 Jacobi-CG" %
            (na, rad, net, seed, scale, levels, info["n_nodes"]))


def cpu_baseline(prob, args):
    """The oracle's whole path on the same molecule (markers, density,
    assembly, Jacobi-CG to the tolerance, potential at the atoms, energy), one
    solve on all host cores, timed."""
    from oracle_lib import Oracle
    o = Oracle(prob)
    t0 = time.perf_counter()
    e, _, it, _ = o.run("cg", args.tol)
    o.phi_on_atoms()
    dt = time.perf_counter() - t0
    o.close()
    return {"value": 1.0 / dt, "unit": "solves/s", "cores": os.cpu_count() or 1, "kind": "port",
            "sample": "one whole solve of the same molecule by the CPU oracle: markers, density, assembly, "
                      "Jacobi-CG to %g (%d iterations), potential at the atoms, energy (%.1f s)" % (args.tol, it, dt),
            "energy_kT": e["sum"]}


def molecule_spec(args):
    """(n_atoms, radius, net charge, seed, levels, scale) of a single-molecule workload."""
    na, rad, net, seed, scale, levels = WORKLOADS[args.workload]
    return (na, rad, net, seed, levels, scale)


def prepare_inputs(specs, outdir, threads=8):
    """Host builds (libpbhost) of the given molecules, saved as numpy arrays,
    one file per molecule: the inputs of the reference arm, made in a process
    of their own so the timed process loads no library of this package."""
    from concurrent.futures import ThreadPoolExecutor

    from cudanextgenpb_b200 import configs
    from oracle_lib import problem_arrays

    def one(item):
        key, (na, rad, net, seed, lv, scale) = item
        prob = configs.make_globular_problem(na, rad, net, seed, scale=scale, levels=lv).build()
        np.savez(os.path.join(outdir, "%s.npz" % key), **problem_arrays(prob))
        prob.close()

    with ThreadPoolExecutor(max_workers=threads) as ex:
        list(ex.map(one, specs.items()))


def reference_inputs(specs, outdir):
    """Runs prepare_inputs for `specs` ({key: spec}) in a subprocess."""
    spec_file = os.path.join(outdir, "specs.json")
    json.dump({k: list(v) for k, v in specs.items()}, open(spec_file, "w"))
    r = subprocess.run([sys.executable, os.path.abspath(__file__), "--prepare-inputs", outdir],
                       capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("input preparation failed: " + r.stderr[-2000:])


def oracle_request(path, tol):
    """The oracle's whole path on one saved molecule: markers, density,
    assembly, Jacobi-CG to tol, potential at the atoms, energy.  Returns
    (seconds, iterations, energy)."""
    from oracle_lib import ArrayProblem, Oracle
    d = dict(np.load(path))
    t0 = time.perf_counter()
    o = Oracle(ArrayProblem(d))
    e, _, it, _ = o.run("cg", tol)
    o.phi_on_atoms()
    dt = time.perf_counter() - t0
    o.close()
    return dt, it, e["sum"]


def run_reference(args, rank, world):
    """The reference arm: the CPU oracle (this package's C++ restatement of
    the reference path; the reference itself cannot be built here) timed on
    the host cores, whole solves with CG run to the tolerance.  Rank 0 alone
    runs; its inputs come from a separate process (prepare_inputs)."""
    if rank != 0:
        return None
    import tempfile
    serve = args.workload in SERVES
    with tempfile.TemporaryDirectory() as tmp:
        if serve:
            per_step = SERVES[args.workload][5]
            specs = serve_specs(args.workload)
            # a step is one request: the first K requests of the timed stream
            picks = serve_picks(args.workload, (args.warmup + args.steps) * per_step)[args.warmup * per_step:]
            timed = [int(k) for k in picks[:args.steps]]
            small = min(range(len(specs)), key=lambda k: specs[k][0])
            warm = [small] * args.warmup
            need = {"m%d" % k: tuple(specs[k]) + (2.0,) for k in set(timed + warm)}
            files = lambda ks: [os.path.join(tmp, "m%d.npz" % k) for k in ks]
            desc = ("the first %d requests of the timed stream, one at a time (pool molecules %s); warm-up: %d "
                    "solves of the smallest pool molecule" % (args.steps, timed, args.warmup))
        else:
            need = {"w": molecule_spec(args), "s": (60, 7.0, -3.0, 60, 1, 2.0)}
            files = lambda ks: [os.path.join(tmp, "%s.npz" % k) for k in ks]
            timed, warm = ["w"] * args.steps, ["s"] * args.warmup
            desc = ("%d whole solves of the molecule; warm-up: %d solves of a 60-atom molecule"
                    % (args.steps, args.warmup))
        t0 = time.time()
        reference_inputs(need, tmp)
        prep_s = time.time() - t0
        for f in files(warm):
            oracle_request(f, args.tol)
        secs, its = [], []
        for f in files(timed):
            dt, it, _ = oracle_request(f, args.tol)
            secs.append(dt)
            its.append(it)
    threads = os.cpu_count() or 1
    total = float(sum(secs))
    v = len(secs) / total
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * total / len(secs),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": args.workload, "cg_iterations": its, "tol": args.tol,
                       "input_preparation_s": prep_s,
                       "what": "CPU oracle (C++ restatement of the reference path, OpenMP on all host cores): "
                               "markers, density, assembly, Jacobi-CG to tol, potential at the atoms, energy; "
                               "meshes built beforehand in a separate process and not timed"},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": threads, "kind": "port",
                             "sample": desc + " (%.1f s timed)" % total},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


BATCHES = {
    # name: (molecules, min atoms, max atoms, seed, surface levels)
    "batch96": (96, 50, 3000, 96, 1),
    "batch16": (16, 50, 600, 16, 1),
}


def build_pool(specs, levels, workers=8):
    """Host problems of a molecule pool, built by a thread pool (the host
    mesh build releases the GIL)."""
    from concurrent.futures import ThreadPoolExecutor

    from cudanextgenpb_b200 import configs

    def one(spec):
        na, rad, net, seed = spec
        return configs.make_globular_problem(na, rad, net, seed, scale=2.0, levels=levels).build()

    t0 = time.time()
    with ThreadPoolExecutor(max_workers=workers) as ex:
        probs = list(ex.map(one, specs))
    log("host pool of %d molecules built in %.1fs" % (len(probs), time.time() - t0))
    return probs


def run_batch(args, rank, world, local):
    """Batched workload: many independent molecules, each with its own octree,
    solved together by the persistent multi-system kernel, against the plain
    path that solves them one at a time.  A step solves every molecule once."""
    import torch

    from cudanextgenpb_b200 import Batch, GpuPath, configs, solver_opts

    if rank != 0 and world > 1:
        return None
    torch.cuda.set_device(local)
    count, lo, hi, seed, levels = BATCHES[args.workload]
    specs = configs.molecule_specs(count, lo, hi, seed)
    probs = build_pool(specs, levels)
    ctxs = [GpuPath(local).load(p) for p in probs]
    n_dof = sum(p.info()["n_nodes"] for p in probs)
    plain_opts = solver_opts("cg", tol=args.tol, max_iter=50000)
    batch_opts = solver_opts("cg", tol=args.tol, max_iter=50000, precision=args.precision, inner_tol=1e-4,
                             check_every=64)

    def setup(g):
        g.create_markers()
        g.create_density_map()
        g.assemble(32, 2048, 4)

    def plain_step():
        out = []
        for g in ctxs:
            setup(g)
            g.solve(plain_opts)
            out.append(g.energy(False)["sum"])
        return out

    b = Batch(local)
    for g in ctxs:
        setup(g)
        b.add(g)

    # the batched path builds the systems and evaluates the energies of its
    # members concurrently (each context has its own stream; the C calls
    # release the GIL), and solves them in one persistent kernel
    from concurrent.futures import ThreadPoolExecutor
    pool = ThreadPoolExecutor(max_workers=max(1, args.workers))

    def batch_step():
        list(pool.map(setup, ctxs))
        stats = b.solve(batch_opts)
        return list(pool.map(lambda g: g.energy(False)["sum"], ctxs)), stats

    def timed(fn, k):
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        r = None
        lat = []
        for _ in range(k):
            a = time.perf_counter()
            r = fn()
            torch.cuda.synchronize()
            lat.append(1e3 * (time.perf_counter() - a))
        return (time.perf_counter() - t0), r, lat

    for _ in range(args.warmup):
        plain_step()
        batch_step()
    clocks = Clocks(local)
    clocks.start()
    t_plain, e_plain, _ = timed(plain_step, args.steps)
    t_batch, (e_batch, stats), lat = timed(batch_step, args.steps)
    ck = clocks.stop()
    err = max(abs(x - y) / max(abs(y), 1e-300) for x, y in zip(e_batch, e_plain))
    value = count * args.steps / t_batch
    plain = count * args.steps / t_plain
    iters = [s.iterations for s in stats.values()]
    pool.shutdown()
    b.close()
    for g in ctxs:
        g.close()
    return {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * t_batch / args.steps,
        "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99))},
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64"
        else "f32-inner/f64", "data": "synthetic",
        "config": {"workload": "%d synthetic molecules, atoms log-uniform in %d-%d (seed %d), own octree each, "
                               "scale 2/A, %d surface level(s); one persistent multi-system CG per step"
                               % (count, lo, hi, seed, levels, ),
                   "n_dof_total": n_dof, "tol": args.tol, "precision": args.precision,
                   "inner_iterations_median": float(np.median(iters)),
                   "plain_solves_per_s": plain, "speedup_vs_plain": value / plain,
                   "max_rel_energy_err_vs_plain": err,
                   "batched_setup_threads": args.workers,
                   "plain_path": "one molecule at a time: set-up, solve, energy",
                   "wall_clock": "host perf_counter around each step after a device synchronize"},
        "clocks": ck,
    }


CHARGES = {
    # name: (n_atoms, net charge, seed, surface levels, charge vectors, titratable sites flipped per vector)
    "charges64": (5000, 0.0, 5000, 1, 64, 8),
}


def run_charges(args, rank, world, local):
    """Many charge vectors on one molecule: each vector flips +-1 e on 8
    random titratable sites of a 5,000-atom synthetic molecule; a step solves
    all 64 through one pbgpu_solve_charges call (one matrix, 64 right-hand
    sides sharing every SpMV), against the plain FP64 path solving them one at
    a time (new charges, density map, right-hand side, solve, energy)."""
    import torch

    from cudanextgenpb_b200 import GpuPath, configs, solve_charges, solver_opts

    if rank != 0 and world > 1:
        return None
    torch.cuda.set_device(local)
    na, net, seed, levels, k, flips = CHARGES[args.workload]
    prob = configs.make_globular_problem(na, configs.radius_for(na), net, seed, scale=2.0, levels=levels)
    g = prob.build_on_gpu(GpuPath(local))
    g.create_markers()
    g.create_density_map()
    g.assemble()
    pos, q, _ = prob.atoms()
    rng = np.random.default_rng(64)
    Q = np.repeat(q[None, :], k, axis=0)
    for j in range(k):
        Q[j, rng.choice(na, size=flips, replace=False)] += rng.choice([-1.0, 1.0], size=flips)
    opts = solver_opts("cg", tol=args.tol, max_iter=50000)
    plain = GpuPath(local)
    prob2 = configs.make_globular_problem(na, configs.radius_for(na), net, seed, scale=2.0, levels=levels)
    prob2.build_on_gpu(plain)

    def plain_all():
        out = []
        for j in range(k):
            plain.set_atoms(pos, Q[j])
            e, _ = plain.run(opts)
            out.append(e["sum"])
        return out

    for _ in range(args.warmup):
        solve_charges(g, Q, opts)
    plain_all()
    torch.cuda.synchronize()
    clocks = Clocks(local)
    clocks.start()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        es, ss = solve_charges(g, Q, opts)
    torch.cuda.synchronize()
    t_multi = time.perf_counter() - t0
    t0 = time.perf_counter()
    ep = plain_all()
    t_plain = time.perf_counter() - t0
    ck = clocks.stop()
    err = max(abs(a["sum"] - b) / abs(b) for a, b in zip(es, ep))
    value = k * args.steps / t_multi
    g.close()
    plain.close()
    return {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_multi / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": "%d charge vectors (+-1 e on %d random sites each, seed 64) on a %d-atom synthetic "
                                   "molecule (net %+g e, seed %d), scale 2/A, %d surface level(s), %d DoF; one "
                                   "multi-right-hand-side solve per step" % (k, flips, na, net, seed, levels, g.n),
                       "plain_solves_per_s": k / t_plain, "speedup_vs_plain_fp64": value / (k / t_plain),
                       "max_rel_energy_err_vs_plain": err, "tol": args.tol,
                       "iterations_max": max(s.iterations for s in ss),
                       "wall_clock": "host perf_counter after a device synchronize"},
            "clocks": ck}


SERVES = {
    # name: (pool size, min atoms, max atoms, seed, surface levels drawn from, requests per step)
    # the request stream: seeded synthetic molecules (atoms log-uniform in
    # [min, max], integer net charges), scale 2/A, each request's mesh built on
    # the GPU as part of serving it
    "serve": (24, 200, 2000, 5, (1, 2), 8),
    # small molecules, one surface level
    "serve_small": (8, 50, 400, 5, (1,), 16),
}


def serve_specs(name):
    """(n_atoms, radius, net charge, seed, surface levels) of the pool's molecules."""
    from cudanextgenpb_b200 import configs
    npool, lo, hi, seed, levels, _ = SERVES[name]
    specs = configs.molecule_specs(npool, lo, hi, seed)
    lv = np.random.default_rng(seed + 1).choice(np.array(levels), size=npool)
    return [(na, rad, net, s, int(l)) for (na, rad, net, s), l in zip(specs, lv)]


def serve_picks(name, n):
    """The pool molecule of each of the first n requests of the stream."""
    npool, _, _, seed = SERVES[name][:4]
    return np.random.default_rng(seed + 2).integers(0, npool, size=n)


class PoolMolecule:
    """A request's payload: the molecule (atoms, charges, radii) and its
    options; the host part of the mesh set-up is only the domain box
    (create_mesh), the rest is built on the GPU (Problem.mesh_build)."""

    def __init__(self, spec):
        from cudanextgenpb_b200 import configs
        na, rad, net, seed, lv = spec
        self.spec = spec
        self.prob = configs.make_globular_problem(na, rad, net, seed, scale=2.0, levels=lv)
        self.build = self.prob.mesh_build()
        self.pos, self.q, self.radius = self.prob.atoms()
        self.model = self.prob.model()
        self.upload_bytes = int(self.pos.nbytes + self.q.nbytes + self.radius.nbytes + 4 * 8 * len(self.q))


def plain_request(g, m, opts):
    """One request through the plain path, one call per reference stage:
    mesh build, markers, density, assembly, FP64 solve, energy."""
    g.build_mesh(m.build)
    g.set_atoms(m.pos, m.q)
    g.set_model(m.model)
    g.create_markers()
    g.create_density_map()
    g.assemble()
    st = g.solve(opts)
    return g.energy(False), st


def serve_stream(srv, reqs, arrivals=None):
    """Submits reqs (all at once, or at `arrivals` seconds after the start) and
    drains the server; returns (seconds, {tag: result}, {tag: latency ms})."""
    t0 = time.perf_counter()
    res, lat = {}, {}
    nxt, n = 0, len(reqs)
    if arrivals is None:
        for r in reqs:
            srv.submit(r)
        nxt = n
    while len(res) < n:
        now = time.perf_counter() - t0
        while nxt < n and arrivals[nxt] <= now:
            srv.submit(reqs[nxt])
            nxt += 1
        for r in srv.progress():
            res[r["tag"]] = r
            lat[r["tag"]] = 1e3 * (time.perf_counter() - t0 - (arrivals[r["tag"]] if arrivals is not None else 0.0))
        if nxt < n and not srv.pending()[0] and not srv.pending()[1]:
            time.sleep(max(0.0, min(arrivals[nxt] - (time.perf_counter() - t0), 0.002)))
    return time.perf_counter() - t0, res, lat


def spmv_roofline(local):
    """The SpMV roofline on the 2,000-atom molecule at 3 surface levels (14.5 M
    DoF, 161 M nonzeros, matrix far larger than L2: the single-molecule FP64
    configuration), plain FP64 CG solves with CUDA events around every SpMV
    launch on the context's stream."""
    from cudanextgenpb_b200 import GpuPath, configs, solver_opts
    na, rad, net, seed, scale, levels = WORKLOADS["mol2000"]
    prob = configs.make_globular_problem(na, rad, net, seed, scale=scale, levels=levels)
    g = prob.build_on_gpu(GpuPath(local))
    g.create_markers()
    g.create_density_map()
    g.assemble(32, 2048, 4)
    opts = solver_opts("cg", tol=1e-8, max_iter=50000)
    g.solve(opts)
    g.set_profiling(True)
    g.reset_counters()
    for _ in range(3):
        st = g.solve(opts)
    cnt = g.counters()
    nnz = info_nnz(g)
    g.close()
    avg = cnt["spmv_ms"] / max(cnt["spmv_launches"], 1)
    peak, kind = measured_peak()
    achieved = cnt["spmv_bytes"] / (avg / 1e3) / 1e9
    tr = spmv_traffic()
    kname = "k_cg_spmv<double, 8>" if os.environ.get("PBGPU_SPMV_PAIRS", "1") != "0" else "k_cg_spmv<double, 4>"
    traffic = None
    if tr and kname in tr.get("kernels", {}):
        traffic = tr["kernels"][kname]["dram_bytes_per_launch"] * (nnz / tr["nnz"])
    return {"kernel": kname + " (SELL-C-sigma SpMV fused with p.Ap)", "bound": "hbm", "achieved": achieved,
            "peak": peak, "unit": "GB/s", "frac": achieved / peak, "peak_kind": peak_kind_text(kind),
            "traffic": traffic, "algorithmic_bytes_per_launch": cnt["spmv_bytes"], "avg_launch_ms": avg,
            "launches_timed": cnt["spmv_launches"],
            "workload": "2,000-atom molecule, 3 surface levels (%d DoF, nnz %d), plain FP64 Jacobi-CG, %d iterations "
                        "per solve, 3 solves" % (g.n, nnz, st.iterations)}


def peak_kind_text(kind):
    return "of measured (MEASURED_PEAKS.json hbm_gbs)" if kind == "measured" else "of fallback"


def oracle_serve_parity(pool, ids, e_plain, e_served, local, tol):
    """Energies of pool molecules `ids` from the CPU oracle (host-built mesh,
    tight CG) against the plain FP64 and served energies of the same molecules,
    and the potential at every node against the oracle's: of the plain FP64
    path and of the served solver (FP32-inner / FP64-refined CG) on the mesh
    built on the GPU (the host's nodes, in the host's order)."""
    from oracle_lib import Oracle
    from cudanextgenpb_b200 import GpuPath, configs, solver_opts
    out = {"molecules": [], "max_rel_err_plain": 0.0, "max_rel_err_served": 0.0,
           "max_phi_rel_l2_plain": 0.0, "max_phi_rel_l2_mixed": 0.0}
    for k in ids:
        na, rad, net, seed, lv = pool[k].spec
        prob = configs.make_globular_problem(na, rad, net, seed, scale=2.0, levels=lv).build()
        o = Oracle(prob)
        oe, ophi, it, rel = o.run("cg", 1e-12)
        o.close()
        prob.close()
        g = GpuPath(local)
        plain_request(g, pool[k], solver_opts("cg", tol=tol, max_iter=50000))
        phi64 = g.phi().copy()
        g.solve(solver_opts("cg", tol=tol, max_iter=50000, precision="mixed", inner_tol=1e-4))
        phim = g.phi().copy()
        g.close()
        nrm = np.linalg.norm(ophi)
        dp = float(np.linalg.norm(phi64 - ophi) / nrm) if phi64.shape == ophi.shape else None
        dm = float(np.linalg.norm(phim - ophi) / nrm) if phim.shape == ophi.shape else None
        ep = abs(e_plain[k] - oe["sum"]) / abs(oe["sum"])
        es = abs(e_served[k] - oe["sum"]) / abs(oe["sum"])
        out["molecules"].append({"atoms": na, "levels": lv, "oracle_kT": oe["sum"], "plain_kT": e_plain[k],
                                 "served_kT": e_served[k], "rel_err_plain": ep, "rel_err_served": es,
                                 "phi_rel_l2_plain": dp, "phi_rel_l2_mixed": dm})
        out["max_rel_err_plain"] = max(out["max_rel_err_plain"], ep)
        out["max_rel_err_served"] = max(out["max_rel_err_served"], es)
        for key, v in (("max_phi_rel_l2_plain", dp), ("max_phi_rel_l2_mixed", dm)):
            out[key] = max(out[key], v) if v is not None and out[key] is not None else None
    return out


def serve_cpu_baseline(pool, picks, tol, budget_s=20.0):
    """The oracle's whole path (markers .. energy, CG to tol) on the stream's
    first requests, one at a time on all host cores, until budget_s of CPU
    time: solves/s of that bounded sample."""
    from oracle_lib import Oracle
    from cudanextgenpb_b200 import configs
    done, t_total, ids = 0, 0.0, []
    for k in picks:
        na, rad, net, seed, lv = pool[k].spec
        prob = configs.make_globular_problem(na, rad, net, seed, scale=2.0, levels=lv).build()
        o = Oracle(prob)
        t0 = time.perf_counter()
        o.run("cg", tol)
        t_total += time.perf_counter() - t0
        o.close()
        prob.close()
        done += 1
        ids.append(int(k))
        if t_total >= budget_s:
            break
    return {"value": done / t_total, "unit": "solves/s", "cores": os.cpu_count() or 1, "kind": "port",
            "sample": "the CPU oracle's markers, density, assembly, Jacobi-CG to %g and energy on the stream's first "
                      "%d requests (pool molecules %s), one at a time, %.1f s; meshes built on the host beforehand "
                      "(not timed)" % (tol, done, ids, t_total)}


def run_serve(args, rank, world, local):
    """The headline: a seeded request stream of synthetic molecules served by
    the continuous-batching server (FP32-inner / FP64-refined solves, whole
    requests on concurrent worker contexts), against the plain FP64 path taking
    the same requests one at a time.  Every request's mesh (initial octree,
    surface refinement, nodes, hanging nodes, ray tables) is built on the GPU
    inside the request.  Replicas under torchrun: every rank serves its own copy
    of the stream on its own GPU."""
    import torch

    from cudanextgenpb_b200 import GpuPath, Server, solver_opts

    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    npool, lo, hi, seed, levels, per_step = SERVES[args.workload]
    specs = serve_specs(args.workload)
    pool = [PoolMolecule(s) for s in specs]
    n_warm, n_req = args.warmup * per_step, args.steps * per_step
    picks = serve_picks(args.workload, n_warm + n_req)
    warm, timed = picks[:n_warm], picks[n_warm:]
    opts64 = solver_opts("cg", tol=args.tol, max_iter=50000)

    def sync_all():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    # the pool's largest molecule (atoms x 4^levels): both arms solve it once
    # before their warm-up, so no context first grows to its size in the
    # timed region
    big = max(range(len(pool)), key=lambda k: pool[k].spec[0] * 4 ** pool[k].spec[4])

    # ---- plain FP64, one request at a time
    g = GpuPath(local)
    size = {}  # pool molecule -> (DoF, nonzeros)
    plain_request(g, pool[big], opts64)
    for k in warm:
        plain_request(g, pool[k], opts64)
        size[int(k)] = (g.n, info_nnz(g))
    g.reset_counters()
    sync_all()
    clocks = Clocks(local)
    clocks.start()
    e_plain, lat_p, it_p = {}, [], []
    t0 = time.perf_counter()
    for k in timed:
        a = time.perf_counter()
        e, st = plain_request(g, pool[k], opts64)
        lat_p.append(1e3 * (time.perf_counter() - a))
        e_plain[int(k)] = e["sum"]
        it_p.append(st.iterations)
        if int(k) not in size:
            size[int(k)] = (g.n, info_nnz(g))
    torch.cuda.synchronize()
    t_plain = max_over_ranks(time.perf_counter() - t0, dist)
    plain_launches = g.counters()["launches"]
    g.close()

    # ---- served: continuous batching of whole requests, FP32-inner solves
    srv = Server(local, tol=args.tol, precision=args.precision, mode=1 if args.server_mode == "concurrent" else 0,
                 workers=args.workers, max_members=args.max_members, steps_per_tick=32, inner_tol=1e-4)

    def requests(ks):
        return [srv.request(pool[k].prob, tag=j, build=pool[k].build) for j, k in enumerate(ks)]

    serve_stream(srv, [srv.request(pool[big].prob, tag=j, build=pool[big].build)
                       for j in range(max(args.workers, 1))])
    serve_stream(srv, requests(warm))
    sync_all()
    l0 = srv.stats()["launches"]
    t_served, res, _ = serve_stream(srv, requests(timed))
    torch.cuda.synchronize()
    t_served = max_over_ranks(t_served, dist)
    served_launches = srv.stats()["launches"] - l0
    # latency at an offered load the server sustains: Poisson arrivals at 70 %
    # of the capacity just measured
    rate = 0.7 * len(timed) / t_served
    arrivals = np.cumsum(np.random.default_rng(seed + 3).exponential(1.0 / rate, size=len(timed)))
    sync_all()
    t_lat, res_lat, lat_s = serve_stream(srv, requests(timed), arrivals)
    srv.close()
    ck = clocks.stop()

    bad = [r for r in list(res.values()) + list(res_lat.values()) if r["status"] != 0]
    e_served = {}
    err_plain = 0.0
    for j, k in enumerate(timed):
        for r in (res[j], res_lat[j]):
            e_served[int(k)] = r["energy"]["sum"]
            err_plain = max(err_plain, abs(r["energy"]["sum"] - e_plain[int(k)]) / abs(e_plain[int(k)]))
    result = None
    if rank == 0:
        value = world * len(timed) / t_served
        plain = world * len(timed) / t_plain
        pct = lambda a: {"p50": float(np.percentile(a, 50)), "p95": float(np.percentile(a, 95)),
                         "p99": float(np.percentile(a, 99))}
        h2d = sum(pool[k].upload_bytes for k in timed)
        # the Krylov iterations' algorithmic bytes over each stream's time: how
        # close the streams run to the HBM bound of their solves alone
        peak, peak_kind = measured_peak()
        b_plain = sum(it * (12 * size[int(k)][1] + 104 * size[int(k)][0]) for it, k in zip(it_p, timed))
        b_served = sum(res[j]["iterations"] * (8 * size[int(k)][1] + 52 * size[int(k)][0])
                       for j, k in enumerate(timed))
        stream_bw = {
            "plain_solve_gbs": b_plain / t_plain / 1e9, "served_solve_gbs": b_served / t_served / 1e9,
            "peak_gbs": peak, "peak_kind": peak_kind_text(peak_kind),
            "served_solve_floor_s": b_served / (peak * 1e9), "served_s": t_served,
            "what": "CG iterations x algorithmic bytes per iteration (FP64: 12 nnz + 104 n; FP32 inner: 8 nnz + "
                    "52 n) summed over the timed requests, divided by the stream's time; mesh build, set-up "
                    "and energy excluded from the bytes but not from the time"}
        # the oracle on the three smallest molecules the stream served (tight solve)
        served_ids = sorted(set(int(k) for k in timed), key=lambda k: pool[k].spec[0])[:3]
        parity = oracle_serve_parity(pool, served_ids, e_plain, e_served, local, args.tol)
        roof = spmv_roofline(local)
        n_dof = [0]
        result = {
            "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * t_served / args.steps,
            "latency_ms": pct(list(lat_s.values())), "higher_is_better": True, "scaling": "weak",
            "vs_baseline": None, "dtype": "f32-inner/f64" if args.precision == "mixed" else "f64",
            "data": "synthetic",
            "config": {
                "workload": "PB request stream: %d requests per step (%d timed) drawn from %d synthetic molecules "
                            "(atoms log-uniform in %d-%d, FCC-lattice subsets, net charge in [-5, 5], seed %d), "
                            "scale 2/A, %s surface level(s); every request's mesh built on the GPU inside it; served "
                            "by %d concurrent worker contexts with %s solves to rel. residual %g, against the plain "
                            "FP64 path one request at a time" % (per_step, len(timed), npool, lo, hi, seed,
                                                                  "/".join(map(str, levels)), args.workers,
                                                                  "FP32-inner/FP64-refined" if args.precision ==
                                                                  "mixed" else "FP64", args.tol),
                "speedup_vs_plain_fp64": value / plain,
                "plain_fp64_solves_per_s": plain,
                "plain_fp64_latency_ms": pct(lat_p),
                "latency_load": "Poisson arrivals at %.1f req/s (70%% of the measured capacity), %d requests; "
                                "latency from arrival to result" % (rate, len(timed)),
                "max_rel_energy_err_served_vs_plain_fp64": err_plain,
                "oracle_parity": parity,
                "stream_bandwidth": stream_bw,
                "failed_requests": len(bad),
                "plain_cg_iterations_median": float(np.median(it_p)),
                "served_iterations_median": float(np.median([r["iterations"] for r in res.values()])),
                "tol": args.tol, "precision": args.precision, "server_mode": args.server_mode,
                "workers": args.workers,
                "plain_gpu_launches": plain_launches,
                "l2": "each request's matrix and vectors are smaller than L2 for most of the pool; requests run "
                      "back to back with no L2 flush, as a server would run them",
                "wall_clock": "host perf_counter around each stream after a device synchronize",
                "warm_up": "the plain context and every worker context first solve the pool's largest molecule, "
                           "then each path takes the warm-up requests (untimed)",
                "parallelism": "replicas (one server per GPU)" if world > 1 else "one GPU",
            },
            "e2e": {"value": value, "unit": "solves/s", "h2d_bytes_per_step": h2d // args.steps,
                    "d2h_bytes_per_step": 96 * per_step,
                    "note": "the same measurement as value: a request is a host-side molecule that the server "
                            "uploads, meshes and solves on the GPU and answers to the host"},
            "roofline": roof,
            "gpu_launches": served_launches,
            "clocks": ck,
        }
        if world == 1 and not args.no_cpu_baseline:
            result["cpu_baseline"] = serve_cpu_baseline(pool, timed, args.tol)
    if dist:
        dist.barrier()
        dist.destroy_process_group()
    return result


def spawn_replicas(n):
    """Re-run this command as n ranks under torchrun on this node (127.0.0.1
    rendezvous on a free port); returns its exit status."""
    import socket
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    cmd = [sys.executable, "-m", "torch.distributed.run", "--nnodes=1", "--nproc-per-node", str(n),
           "--master-addr", "127.0.0.1", "--master-port", str(port), os.path.abspath(__file__)] + sys.argv[1:]
    return subprocess.call(cmd)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="serve",
                    choices=sorted(WORKLOADS) + sorted(BATCHES) + sorted(SERVES) + sorted(CHARGES))
    ap.add_argument("--max-members", type=int, default=64)
    ap.add_argument("--via-batch", action="store_true", help="solve through the persistent multi-system kernel")
    ap.add_argument("--server-mode", default="concurrent", choices=["concurrent", "batched"])
    ap.add_argument("--compare-fp64", action="store_true", help="mixed precision: error against a plain FP64 solve")
    ap.add_argument("--workers", type=int, default=8)
    ap.add_argument("--precision", default=None, choices=["fp64", "mixed"],
                    help="default: mixed for the served stream, fp64 otherwise")
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--chunk", type=int, default=32)
    ap.add_argument("--sigma", type=int, default=2048)
    ap.add_argument("--group", type=int, default=4)
    ap.add_argument("--precond", default="jacobi", choices=["jacobi", "block_jacobi", "none"])
    ap.add_argument("--prepare-inputs", default=None, help=argparse.SUPPRESS)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    if args.prepare_inputs:
        specs = json.load(open(os.path.join(args.prepare_inputs, "specs.json")))
        prepare_inputs({k: tuple(v) for k, v in specs.items()}, args.prepare_inputs)
        return
    args.warmup = max(args.warmup, 3)
    if args.precision is None:
        args.precision = "mixed" if args.workload in SERVES else "fp64"
    if args.gpus > 1 and "WORLD_SIZE" not in os.environ:
        # one process per GPU: start the replicas under torchrun (rank 0 prints the line)
        sys.exit(spawn_replicas(args.gpus))
    rank, world, local = dist_env()
    from cudanextgenpb_b200 import build as b
    if rank == 0:
        b.build_all()
    if args.impl == "reference" and args.workload not in BATCHES and args.workload not in CHARGES:
        res = run_reference(args, rank, world)
    elif args.workload in CHARGES:
        res = run_charges(args, rank, world, local) if args.impl == "ours" else {
            "impl": "reference", "unavailable": "the charge-vector workload is measured against the plain GPU path"}
    elif args.workload in SERVES:
        res = run_serve(args, rank, world, local)
    elif args.workload in BATCHES:
        res = run_batch(args, rank, world, local) if args.impl == "ours" else {
            "impl": "reference", "unavailable": "batched workloads are measured against the plain GPU path"}
    else:
        res = run_ours(args, rank, world, local)
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()

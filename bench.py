"""Benchmark of the PB assemble/solve/energy path (one JSON line on rank 0).

A step is one complete PB solve of one molecule through the GPU path:
create_markers -> create_density_map -> assemble (SELL-C-sigma) -> Krylov solve
-> potential at atoms -> energy.  Default workload (the plain-FP64 2,000-atom
configuration): a seeded synthetic globular molecule, 2,000 atoms on a lattice
subset inside an 18 A sphere, net charge -3 e, mesh_shape 0 at scale 2/A with 3
surface refinement levels, Jacobi-CG to a relative residual of 1e-8.

value   solves/s with mesh, rays and atoms already resident in HBM.
e2e     the same, through the C ABI from pinned host buffers: every step uploads
        the inputs (pbgpu_set_mesh / set_rays / set_atoms / set_model) and reads
        back the potential at the atoms and the energies.
Multi-GPU (torchrun): one process per GPU, each solving its own copy of the
molecule (independent solves, no data-path collective); timing is the max over
ranks.  --impl reference times the CPU restatement of the reference path.
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
# Jacobi-CG iterations to ||r|| <= 1e-8 ||b|| on the large workloads (the same
# count on the GPU and on the CPU oracle: one algorithm, differing only in
# rounding); the CPU arm times a sample of iterations and scales to this count.
# Smaller workloads are solved to convergence on the CPU to find it.
CG_ITERS_1E8 = {"mol2000": 1405, "mol2000l2": 889}


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
    g.set_profiling(True)
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
    g.set_profiling(False)
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
            result["cpu_baseline"] = cpu_baseline(prob, g, int(np.median(iters)), args)
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


def cpu_baseline(prob, g, gpu_iters, args):
    """The oracle's Jacobi-CG on the same assembled system, all host cores: a
    bounded sample of iterations, scaled to solves/s with the GPU's iteration
    count.  Assembly and energy are not timed on the CPU side."""
    from oracle_lib import Oracle
    o = Oracle(prob)
    rp, col, val, rhs = g.system()
    o.set_system(rp, col, val, rhs)
    threads = os.cpu_count() or 1
    it = args.cpu_iters
    t = o.time_cg(it, threads)
    per_iter = t / it
    o.close()
    return {"value": 1.0 / (per_iter * gpu_iters), "unit": "solves/s", "cores": threads, "kind": "port",
            "sample": "%d Jacobi-CG iterations of the CPU oracle on the same %d-DoF system (%.2f s, %.1f ms/iter), "
                      "scaled by the GPU's %d iterations per solve; assembly and energy excluded"
                      % (it, g.n, t, 1e3 * per_iter, gpu_iters)}


def run_reference(args, rank, world):
    """CPU restatement of the reference path (oracle port), rank 0 only."""
    if rank != 0:
        return None
    from oracle_lib import Oracle
    prob = build_problem(args.workload)
    info = prob.info()
    o = Oracle(prob)
    t0 = time.time()
    o.markers()
    o.density()
    o.assemble("rows")
    t_setup = time.time() - t0
    # the energy post-process (its cost does not depend on the potential's values)
    o.set_phi(np.zeros(o.n))
    t0 = time.time()
    o.energy()
    t_setup += time.time() - t0
    # iterations the full solve needs
    if args.ref_iters:
        iters = args.ref_iters
    elif args.tol == 1e-8 and args.workload in CG_ITERS_1E8:
        iters = CG_ITERS_1E8[args.workload]
    else:
        _, iters, _ = o.solve("cg", args.tol)
    threads = os.cpu_count() or 1
    samples = []
    for _ in range(args.warmup):
        o.time_cg(args.cpu_iters, threads)
    for _ in range(args.steps):
        samples.append(o.time_cg(args.cpu_iters, threads) / args.cpu_iters)
    per_iter = float(np.median(samples))
    need = iters
    sec = t_setup + per_iter * need
    v = 1.0 / sec
    return {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": world,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * sec, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": workload_desc(args.workload, info), "n_dof": info["n_nodes"]},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": threads, "kind": "port",
                             "sample": "CPU oracle: markers+density+assembly+energy timed once (%.2f s), %d Jacobi-CG "
                                       "iterations per step timed, scaled to %d iterations per solve"
                                       % (t_setup, args.cpu_iters, need)},
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


SERVES = {
    # name: (pool size, min atoms, max atoms, seed, surface levels, arrivals per s, seconds)
    "serve": (24, 200, 3000, 5, 1, 200.0, 10.0),
    # small molecules, offered faster than either path serves them, so the
    # value is each path's capacity
    "serve_small": (8, 50, 400, 5, 1, 2000.0, 1.0),
}


def run_serve(args, rank, world, local):
    """Serving workload: a seeded Poisson request stream over a pool of
    synthetic molecules, served by the continuous-batching server, against the
    plain FP64 path taking the same requests one at a time.  Latency is from
    each request's arrival time to its result (queueing included)."""
    import torch

    from cudanextgenpb_b200 import GpuPath, Server, configs, solver_opts

    if rank != 0 and world > 1:
        return None
    torch.cuda.set_device(local)
    npool, lo, hi, seed, levels, rate, seconds = SERVES[args.workload]
    specs = configs.molecule_specs(npool, lo, hi, seed)
    probs = build_pool(specs, levels)
    rng = np.random.default_rng(seed)
    arrivals = np.cumsum(rng.exponential(1.0 / rate, size=int(rate * seconds * 1.5)))
    arrivals = arrivals[arrivals < seconds]
    picks = rng.integers(0, npool, size=len(arrivals))
    n_req = len(arrivals)

    # served
    srv = Server(local, tol=args.tol, precision=args.precision, max_members=args.max_members,
                 steps_per_tick=32, inner_tol=1e-4, mode=1 if args.server_mode == "concurrent" else 0,
                 workers=args.workers)
    reqs = [srv.request(p) for p in probs]
    # warm-up: one request of each molecule
    for r in reqs:
        srv.submit(r)
    got = 0
    while got < npool:
        got += len(srv.progress())
    lat_s, e_served = {}, {}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    nxt = 0
    while len(lat_s) < n_req:
        now = time.perf_counter() - t0
        while nxt < n_req and arrivals[nxt] <= now:
            r = srv.request(probs[picks[nxt]], tag=nxt)
            srv.submit(r)
            nxt += 1
        for res in srv.progress():
            k = res["tag"]
            lat_s[k] = 1e3 * (time.perf_counter() - t0 - arrivals[k])
            e_served[k] = res["energy"]["sum"]
        if nxt < n_req and not srv.pending()[0] and not srv.pending()[1]:
            time.sleep(max(0.0, min(arrivals[nxt] - (time.perf_counter() - t0), 0.002)))
    t_served = time.perf_counter() - t0
    srv.close()

    # plain FP64, one at a time, same stream
    g = GpuPath(local)
    plain_opts = solver_opts("cg", tol=args.tol, max_iter=50000)
    e_plain = {}
    for k in range(npool):
        g.load(probs[k])
        g.run(plain_opts)
    lat_p = {}
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    for k in range(n_req):
        now = time.perf_counter() - t0
        if arrivals[k] > now:
            time.sleep(arrivals[k] - now)
        g.load(probs[picks[k]])
        e, _ = g.run(plain_opts)
        e_plain[k] = e["sum"]
        lat_p[k] = 1e3 * (time.perf_counter() - t0 - arrivals[k])
    t_plain = time.perf_counter() - t0
    g.close()
    err = max(abs(e_served[k] - e_plain[k]) / max(abs(e_plain[k]), 1e-300) for k in range(n_req))
    ls = np.array([lat_s[k] for k in range(n_req)])
    lp = np.array([lat_p[k] for k in range(n_req)])
    value = n_req / t_served
    plain = n_req / t_plain
    pct = lambda a: {"p50": float(np.percentile(a, 50)), "p95": float(np.percentile(a, 95)),
                     "p99": float(np.percentile(a, 99))}
    return {
        "metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": 1, "steps": n_req, "warmup": npool,
        "ms_per_step": 1e3 * t_served / n_req, "latency_ms": pct(ls), "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "f32-inner/f64", "data": "synthetic",
        "config": {"workload": "Poisson stream %.0f req/s for %.0f s (seed %d) over %d synthetic molecules, atoms "
                               "log-uniform in %d-%d, scale 2/A, %d surface level(s); continuous-batching server"
                               % (rate, seconds, seed, npool, lo, hi, levels),
                   "requests": n_req, "tol": args.tol, "precision": args.precision,
                   "max_members": args.max_members, "server_mode": args.server_mode, "workers": args.workers,
                   "plain_solves_per_s": plain, "plain_latency_ms": pct(lp), "speedup_vs_plain": value / plain,
                   "max_rel_energy_err_vs_plain": err,
                   "wall_clock": "host perf_counter; latency from each request's scheduled arrival"},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--workload", default="mol2000", choices=sorted(WORKLOADS) + sorted(BATCHES) + sorted(SERVES))
    ap.add_argument("--max-members", type=int, default=64)
    ap.add_argument("--via-batch", action="store_true", help="solve through the persistent multi-system kernel")
    ap.add_argument("--server-mode", default="concurrent", choices=["concurrent", "batched"])
    ap.add_argument("--compare-fp64", action="store_true", help="mixed precision: error against a plain FP64 solve")
    ap.add_argument("--workers", type=int, default=8)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "mixed"])
    ap.add_argument("--tol", type=float, default=1e-8)
    ap.add_argument("--chunk", type=int, default=32)
    ap.add_argument("--sigma", type=int, default=2048)
    ap.add_argument("--group", type=int, default=4)
    ap.add_argument("--precond", default="jacobi", choices=["jacobi", "block_jacobi", "none"])
    ap.add_argument("--cpu-iters", type=int, default=30)
    ap.add_argument("--ref-iters", type=int, default=0)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    args = ap.parse_args()
    args.warmup = max(args.warmup, 3)
    rank, world, local = dist_env()
    from cudanextgenpb_b200 import build as b
    if rank == 0:
        b.build_all()
    if args.workload in SERVES:
        res = run_serve(args, rank, world, local) if args.impl == "ours" else {
            "impl": "reference", "unavailable": "the serving workload is measured against the plain GPU path"}
    elif args.workload in BATCHES:
        res = run_batch(args, rank, world, local) if args.impl == "ours" else {
            "impl": "reference", "unavailable": "batched workloads are measured against the plain GPU path"}
    elif args.impl == "reference":
        res = run_reference(args, rank, world)
    else:
        res = run_ours(args, rank, world, local)
    if rank == 0 and res is not None:
        print(json.dumps(res), flush=True)


if __name__ == "__main__":
    main()

"""Benchmark: Tet10 PCG solve time at rel-res 1e-8 on one B200 (per rank).

Workload (the configuration the headline metric is quoted on): steady thermal
diffusion on the 128x128x128-hex ImprovedMeshGenerator cube (12,582,912 Tet10
elements, 16,974,593 DOFs), domain 1000x1000x600, per-element conductivity
ln k_e ~ N(ln 3, 0.5^2) (seed 1001), Q = 1e-6, T = 1280 at z = 0 and T = 0 at
z = 600, Jacobi-PCG to relative residual 1e-8 with the mixed-precision
matrix-free solver (FP32 operator and PCG, FP64 residual refresh and update).
Synthetic seeded inputs; every input is larger than L2 (126 MB), so no flush.

One "step" is one full solve f_bc -> u on device-resident inputs; `value` is
seconds per solve for the whole job (timed region / (steps * ranks)). The line
also carries the plain-FP64 GPU solve time, the mixed/FP64 speed-up, the
adjoint/forward time ratio on the 48x48x32 inversion configuration, the
end-to-end time through the C ABI with host buffers, the roofline of the
persistent PCG kernel and the CPU baseline (the reference's serial Jacobi-CG
restated in C++, run on the same 128^3 system for a bounded number of
iterations and scaled to the iteration count of the FP64 solve).

Usage: python bench.py [--gpus N] [--steps K] [--warmup W] [--impl reference]
Multi-GPU: launched by torchrun, one independent replica per GPU ("replicas
only": the path has no exchange step at one GPU per solve).
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

from geo_simulator_b200.kernel_timing import patch_pcg_bytes, update_bytes  # noqa: E402

# Iterations of the FP64 Jacobi-PCG (the reference algorithm) to rel-res 1e-8 on the
# n^3 log-normal-k system, measured on the GPU by this repository's FP64 solver
# (same loop, same stopping rule). The reference arm times its per-iteration
# cost on the host and scales by this count, so it never touches the GPU.
FP64_ITERS = {128: 1050}

METRIC = "Tet10 PCG solve time @rel-res 1e-8: mixed vs FP64 GPU; adjoint/forward ratio"
LX, LY, LZ = 1000.0, 1000.0, 600.0
Q = 1e-6


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


def thermal_inputs(n, seed=1001, sigma=0.5, nz=None):
    """Host inputs of the thermal configuration (mesh, k_e, Dirichlet mask/values)."""
    from geo_simulator_b200 import ImprovedMeshGenerator
    from geo_simulator_b200.fields import lognormal_field
    mesh = ImprovedMeshGenerator.generate_cube(n, n, nz or n, LX, LY, LZ)
    k_e = lognormal_field(seed, mesh.num_elements(), np.log(3.0), sigma)
    z = mesh.nodes[:, 2]
    bottom = np.abs(z) < 1.0
    top = (~bottom) & (np.abs(z - LZ) < 1.0)
    mask = (bottom | top).astype(np.uint8)
    vals = np.where(bottom, 1280.0, 0.0)
    return mesh, k_e, mask, vals


def apply_bytes(E, N, s):
    """Algorithmic bytes of one thermal matrix-free apply (int32 connectivity, k_e,
    SoA coordinates, x read, y write, Dirichlet bitmask)."""
    return E * (10 * 4 + s) + N * (3 * s + s + s) + N / 8


def solve_bytes(E, N, iters, nupd):
    """Algorithmic bytes of one mixed solve: per FP32 PCG iteration one patch-kernel
    and one node-update launch; per FP64 refresh one FP64 apply plus 4 FP64 streams."""
    return (iters * (patch_pcg_bytes(E, N, 4) + update_bytes(N, 4))
            + nupd * (apply_bytes(E, N, 8) + 4 * N * 8))


# DRAM bytes (read + write) per element of one FP32 PCG-mode patch-kernel launch,
# measured by ncu (dram__bytes_read.sum + dram__bytes_write.sum) on the bench's
# 128^3 cube (12,582,912 elements: 1008.9 MB per launch).
PATCH_PCG_F32_DRAM_BYTES_PER_ELEMENT = 80.18


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled during the timed region."""

    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", delete=False, suffix=".csv")
        self.p = None

    def start(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                                       "-lms", "200", "-i", str(self.device)], stdout=self.f,
                                      stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None

    def stop(self):
        if self.p is None:
            return None
        time.sleep(0.25)
        self.p.terminate()
        try:
            self.p.wait(timeout=5)
        except Exception:
            self.p.kill()
        self.f.flush()
        self.f.seek(0)
        rows = [r.split(",") for r in self.f.read().strip().splitlines() if r.count(",") >= 8]
        if not rows:
            return None
        sm = [float(r[1]) for r in rows if r[1].strip().replace(".", "").isdigit()]
        smax = [float(r[2]) for r in rows if r[2].strip().replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].strip() == "Active"})
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": reasons, "samples": len(rows)}


def dist_setup(args):
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl" if args.impl == "ours" else "gloo", timeout=datetime.timedelta(seconds=600))
        pg = dist
    return ws, rank, local, pg


def max_over_ranks(v, pg, device):
    if pg is None:
        return v
    import torch
    t = torch.tensor([v], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def barrier(pg, device):
    if pg is not None:
        import torch
        pg.barrier(device_ids=[device]) if torch.cuda.is_available() else pg.barrier()


# --------------------------------------------------------------------------- CPU baseline
def cpu_reference_sample(n, fp64_iters, sample_iters, system=None):
    """The reference's serial Jacobi-CG (iterative.rs:46-119, restated in C++) on the
    same n^3 K_bc, built on the host cores by the oracle (element matrices of
    element.rs:23-61, CSR with sprs semantics, Dirichlet elimination of
    assembly.rs:168-230), timed for `sample_iters` iterations and scaled to
    `fp64_iters`. Returns (seconds per solve, info, system)."""
    from oracle import oracle as orc
    if system is None:
        mesh, k_e, mask, vals = thermal_inputs(n)
        system = orc.ThermalSystem(mesh.nodes, mesh.elements.astype(np.int64), k_e, Q, mask, vals)
    _, st = system.cg(sample_iters, 1e-8)
    per_it = st.solve_time / max(st.iterations, 1)
    return per_it * fp64_iters, {"per_iteration_s": per_it, "nnz": system.nnz,
                                 "sample_iterations": sample_iters}, system


# --------------------------------------------------------------------------- our arm
def run_ours(args, ws, rank, local, pg):
    import torch

    import geo_simulator_b200 as geo
    from geo_simulator_b200 import _native as N
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    n = args.size
    mesh, k_e, mask, vals = thermal_inputs(n)
    E, Nn = mesh.num_elements(), mesh.num_nodes()
    ctx = geo.Context(local)
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    dm = geo.DofManager(Nn, 1)
    idx = np.nonzero(mask)[0]
    dm.set_dirichlet(idx, vals[idx])
    op = geo.ThermalOperator(mesh, dm, k_e, ctx)
    f = torch.empty(Nn, dtype=torch.float64, device=dev)
    ctx.check(N.lib().geo_assemble_thermal_load(ctx.h, mesh.handle(ctx), dm.handle(ctx), Q, f.data_ptr()))
    fb = op.lift_rhs(f)
    mixed = geo.ConjugateGradient().with_tolerance(1e-8).with_max_iterations(20000).with_precision("mixed")
    fp64 = geo.ConjugateGradient().with_tolerance(1e-8).with_max_iterations(20000)

    def timed(solver, steps, collect):
        barrier(pg, local)
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        out = None
        for _ in range(steps):
            out = op.solve(fb, solver)
            collect.append(out[1])
        e1.record(stream)
        torch.cuda.synchronize()
        barrier(pg, local)
        return e0.elapsed_time(e1) / 1e3, out[0]

    for _ in range(args.warmup):
        op.solve(fb, mixed)
    clocks = ClockSampler(local)
    clocks.start()
    st_mixed = []
    t_mixed, x_mixed = timed(mixed, args.steps, st_mixed)
    clk = clocks.stop()
    t_mixed = max_over_ranks(t_mixed, pg, dev)
    ms_per_step = 1e3 * t_mixed / args.steps
    value = t_mixed / (args.steps * ws)
    iters = st_mixed[-1].iterations
    nupd = st_mixed[-1].fp64_residual_updates
    kern = statistics.mean(s.solve_time for s in st_mixed)

    extras = {}
    if not args.quick:
        # plain FP64 GPU path on the same system
        op.solve(fb, fp64)
        st64 = []
        t64, x64 = timed(fp64, max(1, min(args.steps, 2)), st64)
        t64 /= len(st64)
        # accuracy of the mixed solution: true FP64 residual, distance to the FP64
        # solution at the same tolerance, and both distances to an FP64 solution
        # converged to rel-res 1e-12 (each 1e-8 solve carries its own error)
        r = fb - op.apply(x_mixed)
        r64 = fb - op.apply(x64)
        xc, _ = op.solve(fb, geo.ConjugateGradient().with_tolerance(1e-12).with_max_iterations(50000))
        nrm = lambda v: float(torch.linalg.norm(v))
        extras.update({
            "fp64_solve_s": t64,
            "fp64_iterations": st64[-1].iterations,
            "mixed_speedup_vs_fp64": t64 / (ms_per_step / 1e3),
            "mixed_true_relative_residual": nrm(r) / nrm(fb),
            "fp64_true_relative_residual": nrm(r64) / nrm(fb),
            "mixed_vs_fp64_solution_rel_l2": nrm(x_mixed - x64) / nrm(x64),
            "mixed_vs_converged_rel_l2": nrm(x_mixed - xc) / nrm(xc),
            "fp64_vs_converged_rel_l2": nrm(x64 - xc) / nrm(xc),
        })
        del x64, r, r64, xc
    # end to end through the C ABI with pinned host buffers: mesh + DOFs + k_e up,
    # operator set-up, load, lift, mixed solve, solution down
    e2e = run_e2e(ctx, stream, mesh, k_e, mask, vals, args, dev) if not args.quick else None
    if not args.quick and rank == 0:
        extras.update(adjoint_ratio(ctx, args))
        extras["csr_vs_matfree_64"] = csr_vs_matfree(ctx)
        extras["elasticity_48x48x24"] = elasticity_config(ctx)
        extras["neumann_128"] = neumann_timing(ctx, mesh)
        extras["maxwell_step_48x48x24"] = maxwell_step(ctx)
        extras["meshgen_128"] = meshgen_timing(ctx, n)
        extras["vtu_128"] = vtu_output(ctx, mesh, x_mixed)

    # dominant kernel: the FP32 patch kernel in PCG mode, timed launch by launch with
    # CUDA events on the context stream right after the timed region
    kt_iters = 50
    pms, ums = C.c_double(), C.c_double()
    ctx.check(N.lib().geo_op_time_pcg_kernels(op.h, fb.data_ptr(), N.PRECISION_MIXED, kt_iters,
                                              C.byref(pms), C.byref(ums)))
    patch_s, update_s = pms.value / 1e3, ums.value / 1e3
    hbm, peak_kind = peaks()
    pbytes = patch_pcg_bytes(E, Nn, 4)
    ubytes = update_bytes(Nn, 4)
    achieved = pbytes / patch_s / 1e9
    traffic = (PATCH_PCG_F32_DRAM_BYTES_PER_ELEMENT * E) if PATCH_PCG_F32_DRAM_BYTES_PER_ELEMENT else None
    abytes = solve_bytes(E, Nn, iters, nupd)
    line = {
        "metric": METRIC, "value": value, "unit": "s", "n_gpus": ws, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": ms_per_step, "higher_is_better": False, "scaling": "weak", "vs_baseline": None,
        "dtype": "f32 inner / f64 refresh", "data": "synthetic (seeded ImprovedMeshGenerator cube, log-normal k)",
        "config": {"workload": f"thermal Tet10 cube {n}^3 hexes, {E} elements, {Nn} DOFs, ln k ~ N(ln 3, 0.5^2), "
                               "mixed-precision matrix-free Jacobi-PCG to rel-res 1e-8",
                   "elements": E, "dofs": Nn, "parallelism": f"replicas x{ws}",
                   "l2": "inputs larger than L2 (no flush)"},
        "iterations": iters, "fp64_residual_updates": nupd,
        "dofs_per_s": Nn * ws / (t_mixed / args.steps),
        "pcg_iterations_per_s": iters / (t_mixed / args.steps),
        "gpu_launches": int(sum(s_.kernel_launches for s_ in st_mixed)),
        "roofline": {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "traffic": traffic, "peak_kind": peak_kind,
                     "kernel": "k_patch<ThermalK<float,1>, float, MODE_PCG, 2, 0> (halo slots in shared memory)",
                     "algorithmic_bytes_per_launch": pbytes, "launch_s": patch_s,
                     "timing": f"CUDA events between launches, {kt_iters} PCG iterations after the timed region",
                     "node_update": {"kernel": "k_pcg_update_halo<float, true>", "launch_s": update_s,
                                     "algorithmic_bytes_per_launch": ubytes,
                                     "achieved": ubytes / update_s / 1e9,
                                     "frac": ubytes / update_s / 1e9 / hbm},
                     "solve": {"algorithmic_bytes": abytes, "device_s": kern,
                               "achieved": abytes / kern / 1e9, "frac": abytes / kern / 1e9 / hbm}},
        "clocks": clk,
    }
    line.update(extras)
    if e2e is not None:
        line["e2e"] = e2e
    if rank == 0 and ws == 1 and not args.no_cpu_baseline:
        fp64_iters = extras.get("fp64_iterations", iters)
        v, info, _ = cpu_reference_sample(n, fp64_iters, args.cpu_iters)
        line["cpu_baseline"] = {
            "value": v, "unit": "s", "cores": 1, "kind": "port",
            "sample": f"reference serial Jacobi-CG (C++ restatement) on the same {n}^3 K_bc, "
                      f"{args.cpu_iters} iterations timed ({info['per_iteration_s']:.3f} s/iteration, "
                      f"nnz {info['nnz']}), scaled to the FP64 iteration count {fp64_iters}"}
    return line


def run_e2e(ctx, stream, mesh, k_e, mask, vals, args, dev):
    import torch

    from geo_simulator_b200 import _native as N
    L = N.lib()
    pin = lambda a: torch.from_numpy(np.ascontiguousarray(a)).pin_memory()
    xyz_h, conn_h = pin(mesh.nodes), pin(mesh.elements)
    k_h, mask_h, vals_h = pin(k_e), pin(mask), pin(vals)
    u_h = torch.empty(mesh.num_nodes(), dtype=torch.float64).pin_memory()
    opts = N.default_opts()
    opts.tolerance = 1e-8
    opts.max_iterations = 20000
    opts.precision = N.PRECISION_MIXED
    steps = max(1, args.e2e_steps)
    times = []
    for it in range(steps + 1):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        m, d, op = C.c_void_p(), C.c_void_p(), C.c_void_p()
        ctx.check(L.geo_mesh_create(ctx.h, mesh.num_nodes(), xyz_h.data_ptr(), mesh.num_elements(),
                                    conn_h.data_ptr(), C.byref(m)))
        ctx.check(L.geo_dofs_create(ctx.h, mesh.num_nodes(), 1, mask_h.data_ptr(), vals_h.data_ptr(), C.byref(d)))
        ctx.check(L.geo_thermal_operator_create(ctx.h, m, d, k_h.data_ptr(), 0.0, C.byref(op)))
        f = torch.empty(mesh.num_nodes(), dtype=torch.float64, device=dev)
        ctx.check(L.geo_assemble_thermal_load(ctx.h, m, d, Q, f.data_ptr()))
        st = N.SolverStatsC()
        ctx.check(L.geo_forward(op, f.data_ptr(), C.byref(opts), u_h.data_ptr(), C.byref(st)))
        e1.record(stream)
        torch.cuda.synchronize()
        L.geo_op_destroy(op)
        L.geo_dofs_destroy(d)
        L.geo_mesh_destroy(m)
        del f
        if it > 0:  # first call pays lazy module loading
            times.append(e0.elapsed_time(e1) / 1e3)
    h2d = (xyz_h.numel() * 8 + conn_h.numel() * 4 + k_h.numel() * 8 + mask_h.numel() + vals_h.numel() * 8)
    return {"value": statistics.median(times), "unit": "s", "h2d_bytes_per_step": int(h2d),
            "d2h_bytes_per_step": int(u_h.numel() * 8), "steps": steps,
            "includes": "mesh/DOF/k upload, GPU patch build, qdata, load, Dirichlet lift, mixed solve, u download"}


def adjoint_ratio(ctx, args):
    """Forward vs adjoint-gradient time on the 48x48x32 inversion configuration."""
    import torch

    import geo_simulator_b200 as geo
    from geo_simulator_b200.fields import choice_distinct, lognormal_field
    mesh, _, mask, vals = thermal_inputs(48, nz=32)
    k_e = lognormal_field(2001, mesh.num_elements(), np.log(3.0), 0.3)
    dm = geo.DofManager(mesh.num_nodes(), 1)
    idx = np.nonzero(mask)[0]
    dm.set_dirichlet(idx, vals[idx])
    op = geo.ThermalOperator(mesh, dm, k_e, ctx)
    f = geo.Assembler.assemble_thermal_load(mesh, dm, Q, ctx)
    solver = geo.ConjugateGradient().with_tolerance(1e-8).with_max_iterations(20000).with_precision("mixed")
    free = np.nonzero(mask == 0)[0]
    obs = free[choice_distinct(2003, free.size, 1000)]
    u, _ = op.forward(f, solver)
    that = u + 1.0
    g = np.zeros_like(u)
    g[obs] = u[obs] - that[obs]
    reps = 5
    op.forward(f, solver)  # warm-up of each timed call
    op.vjp(g, u=u, solver=solver)
    op.vjp(g, u=None, f=f, solver=solver)
    t0 = time.perf_counter()
    for _ in range(reps):
        u, sf = op.forward(f, solver)
    tf = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        grad, sa = op.vjp(g, u=u, solver=solver)
    ta = (time.perf_counter() - t0) / reps
    t0 = time.perf_counter()
    for _ in range(reps):
        grad, sr = op.vjp(g, u=None, f=f, solver=solver)
    tr = (time.perf_counter() - t0) / reps
    # the adjoint right-hand side (point residuals at the observation nodes) needs more
    # PCG iterations to the same relative tolerance than the smooth forward load; the
    # per-iteration cost is the same
    return {"adjoint_forward_ratio": ta / tf, "adjoint_recompute_forward_ratio": tr / tf,
            "adjoint_config": "48x48x32 hexes (442,368 elements, 611,585 DOFs), ln k ~ N(ln 3, 0.3^2), "
                              "1000 observation nodes, mixed precision, host-timed calls",
            "forward_s": tf, "adjoint_s": ta, "forward_iterations": sf.iterations,
            "adjoint_iterations": sa.iterations,
            "adjoint_forward_per_iteration_ratio": (ta / max(1, sa.iterations)) / (tf / max(1, sf.iterations))}


def _host(v):
    """numpy view of a host array or a copy of a device tensor."""
    return v.detach().cpu().numpy() if hasattr(v, "detach") else np.asarray(v)


def _device_timed(ctx, fn, reps=1):
    """Runs fn() reps times between CUDA events on the context stream; seconds per call."""
    import torch
    dev = torch.device("cuda", torch.cuda.current_device())
    stream = torch.cuda.ExternalStream(ctx.stream_handle(), device=dev)
    torch.cuda.synchronize()
    e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    e0.record(stream)
    out = None
    for _ in range(reps):
        out = fn()
    e1.record(stream)
    torch.cuda.synchronize()
    return e0.elapsed_time(e1) / 1e3 / reps, out


def csr_vs_matfree(ctx):
    """64^3 cube, uniform k = 3: plain FP64 matrix-free PCG vs FP64 PCG on the
    assembled CSR (assembly + Dirichlet elimination timed separately)."""
    import torch

    import geo_simulator_b200 as geo
    mesh, _, mask, vals = thermal_inputs(64)
    dm = geo.DofManager(mesh.num_nodes(), 1)
    idx = np.nonzero(mask)[0]
    dm.set_dirichlet(idx, vals[idx])
    f = geo.Assembler.assemble_thermal_load(mesh, dm, Q, ctx)
    dev = torch.device("cuda", torch.cuda.current_device())
    fd = torch.from_numpy(f).to(dev)
    cg = geo.ConjugateGradient().with_tolerance(1e-8).with_max_iterations(20000)
    geo.Assembler.assemble_thermal_stiffness_parallel(mesh, dm, 3.0, ctx)  # warm (inverse map, pattern)
    t_asm, (Kb, fb) = _device_timed(ctx, lambda: geo.Assembler.apply_dirichlet_bcs(
        geo.Assembler.assemble_thermal_stiffness_parallel(mesh, dm, 3.0, ctx), fd, dm, ctx))
    cg.solve(Kb, fb)
    t_csr, (x_csr, st_csr) = _device_timed(ctx, lambda: cg.solve(Kb, fb), 2)
    op = geo.ThermalOperator(mesh, dm, 3.0, ctx)
    op.solve(fb, cg)
    t_mf, (x_mf, st_mf) = _device_timed(ctx, lambda: op.solve(fb, cg), 2)
    return {"config": "64^3 hexes (1,572,864 elements, 2,146,689 DOFs), k = 3, Jacobi-PCG to rel-res 1e-8, FP64",
            "csr_nnz": Kb.nnz(), "csr_assembly_and_bc_s": t_asm, "csr_pcg_s": t_csr,
            "csr_iterations": st_csr.iterations, "matfree_pcg_s": t_mf, "matfree_iterations": st_mf.iterations,
            "matfree_speedup_vs_csr_pcg": t_csr / t_mf,
            "solution_rel_l2": float(np.linalg.norm(_host(x_mf) - _host(x_csr)) / np.linalg.norm(_host(x_csr)))}


def elasticity_config(ctx):
    """48x48x24 hexes of 100 x 100 x 50 km, ln E_e ~ N(ln 1e11, 0.3^2) (seed 3001),
    nu = 0.25, rho = 3300, fixed base, roller sides: mixed and FP64 matrix-free
    solves and the adjoint dJ/d(ln E_e) of a surface u_z misfit at 500 seeded
    top nodes (seed 3002)."""
    import geo_simulator_b200 as geo
    from geo_simulator_b200.fields import choice_distinct, lognormal_field
    lx, ly, lz = 100e3, 100e3, 50e3
    mesh = geo.ImprovedMeshGenerator.generate_cube(48, 48, 24, lx, ly, lz)
    N = mesh.num_nodes()
    x, y, z = mesh.nodes[:, 0], mesh.nodes[:, 1], mesh.nodes[:, 2]
    mask = np.zeros(3 * N, np.uint8)
    base = np.nonzero(np.abs(z) < 1.0)[0]
    for c in range(3):
        mask[3 * base + c] = 1
    mask[3 * np.nonzero((np.abs(x) < 1.0) | (np.abs(x - lx) < 1.0))[0]] = 1
    mask[3 * np.nonzero((np.abs(y) < 1.0) | (np.abs(y - ly) < 1.0))[0] + 1] = 1
    dm = geo.DofManager(N, 3)
    idx = np.nonzero(mask)[0]
    dm.set_dirichlet(idx, np.zeros(idx.size))
    E_e = lognormal_field(3001, mesh.num_elements(), np.log(1e11), 0.3)
    op = geo.ElasticityOperator(mesh, dm, geo.IsotropicElasticity(1e11, 0.25), E_e, ctx)
    f = geo.Assembler.assemble_gravity_load(mesh, dm, 3300.0, [0.0, 0.0, -9.81], ctx)
    mixed = geo.ConjugateGradient().with_tolerance(1e-8).with_max_iterations(50000).with_precision("mixed")
    fp64 = geo.ConjugateGradient().with_tolerance(1e-8).with_max_iterations(50000)
    op.forward(f, mixed)
    tf, (u, sf) = _device_timed(ctx, lambda: op.forward(f, mixed))
    t64, (u64, s64) = _device_timed(ctx, lambda: op.forward(f, fp64))
    top = np.nonzero(np.abs(z - lz) < 1.0)[0]
    obs = 3 * top[choice_distinct(3002, top.size, 500)] + 2
    g = np.zeros_like(u)
    g[obs] = u[obs] - (u[obs] + 1e-3)
    ta, (grad, sa) = _device_timed(ctx, lambda: op.vjp(g, u=u, solver=mixed))
    return {"config": "48x48x24 hexes (331,776 elements, 1,383,123 DOFs), mixed matrix-free PCG to rel-res 1e-8",
            "mixed_forward_s": tf, "mixed_iterations": sf.iterations, "fp64_forward_s": t64,
            "fp64_iterations": s64.iterations, "mixed_speedup_vs_fp64": t64 / tf,
            "mixed_vs_fp64_rel_l2": float(np.linalg.norm(u - u64) / np.linalg.norm(u64)),
            "adjoint_s": ta, "adjoint_forward_ratio": ta / tf, "adjoint_converged": bool(sa.converged)}


def neumann_timing(ctx, mesh):
    """Neumann flux on the top face of the 128^3 cube: GPU boundary-face detection
    (find_boundary_faces) and the deterministic apply_neumann_bcs, host-timed."""
    import geo_simulator_b200 as geo
    top = np.abs(mesh.nodes[:, 2] - LZ) < 1.0
    f = np.zeros(mesh.num_nodes())
    geo.Assembler.find_boundary_faces(mesh, top, ctx)
    t0 = time.perf_counter()
    faces = geo.Assembler.find_boundary_faces(mesh, top, ctx)
    t1 = time.perf_counter()
    geo.Assembler.apply_neumann_bcs(mesh, f, (faces, 0.05), ctx)
    t2 = time.perf_counter()
    return {"faces": int(faces.shape[0]), "find_boundary_faces_s": t1 - t0, "apply_neumann_s": t2 - t1,
            "total_flux": float(f.sum()), "expected_total_flux": 0.05 * LX * LY}


def meshgen_timing(ctx, n):
    """ImprovedMeshGenerator::generate_cube at n^3 hexes: the host generator plus the
    upload into a device mesh, against geo_mesh_generate_cube building the device
    mesh in place (device time includes its allocations). The device mesh is copied
    out once and compared with the host arrays bit for bit."""
    import geo_simulator_b200 as geo
    t0 = time.perf_counter()
    hm = geo.ImprovedMeshGenerator.generate_cube(n, n, n, LX, LY, LZ)
    t1 = time.perf_counter()
    hm.handle(ctx)
    t2 = time.perf_counter()
    geo.ImprovedMeshGenerator.generate_cube_device(n, n, n, LX, LY, LZ, ctx)  # warm-up
    reps = 3
    t3 = time.perf_counter()
    for _ in range(reps):
        dm = geo.ImprovedMeshGenerator.generate_cube_device(n, n, n, LX, LY, LZ, ctx)
        del dm
    t4 = time.perf_counter()
    dev_s, dm = _device_timed(ctx, lambda: geo.ImprovedMeshGenerator.generate_cube_device(n, n, n, LX, LY, LZ, ctx))
    same = bool(np.array_equal(dm.elements, hm.elements)
                and np.array_equal(dm.nodes.view(np.uint64), hm.nodes.view(np.uint64)))
    out_bytes = 24 * dm.num_nodes() + 40 * dm.num_elements()
    return {"nodes": dm.num_nodes(), "elements": dm.num_elements(),
            "host_generate_s": t1 - t0, "host_upload_s": t2 - t1,
            "device_generate_wall_s": (t4 - t3) / reps, "device_generate_events_s": dev_s,
            "speedup_vs_host_generate_and_upload": (t2 - t0) / ((t4 - t3) / reps),
            "device_mesh_bytes": out_bytes, "bit_exact_vs_host": same}


def vtu_output(ctx, mesh, temperature):
    """VtkWriter::write_vtu of the 128^3 mesh with the mixed-precision temperature
    solution as its point field: the GPU render into a device buffer (CUDA events on
    the context stream) and the streamed write of the same text to a file in the
    system temp directory (wall clock, file removed afterwards)."""
    import tempfile

    import geo_simulator_b200 as geo
    from geo_simulator_b200.kernel_timing import render_device
    mesh.field_data.add_field(geo.ScalarField("Temperature", temperature))
    try:
        size, dev_s = render_device(ctx, mesh)
        fd, path = tempfile.mkstemp(suffix=".vtu")
        os.close(fd)
        try:
            t0 = time.perf_counter()
            geo.VtkWriter.write_vtu(mesh, path, ctx)
            wall = time.perf_counter() - t0
        finally:
            os.remove(path)
    finally:
        mesh.field_data.scalar_fields.pop("Temperature", None)
    return {"bytes": size, "render_device_s": dev_s, "render_gbs": size / dev_s / 1e9,
            "write_file_s": wall, "write_file_gbs": size / wall / 1e9}


def maxwell_step(ctx):
    """One backward-Euler step of Maxwell viscoelasticity on the 48x48x24 half-space
    (gravity, fixed base, roller sides, E = 1e11, nu = 0.25, mu = 1e19, dt = tau/10):
    the reference's step (re-assemble K and f_history, CSR Jacobi-PCG, FP64) and the
    step with a resident matrix-free operator (mixed precision), both followed by the
    stress update. Rel-res 1e-8."""
    import geo_simulator_b200 as geo
    lx, ly, lz = 100e3, 100e3, 50e3
    mesh = geo.ImprovedMeshGenerator.generate_cube(48, 48, 24, lx, ly, lz)
    N = mesh.num_nodes()
    x, y, z = mesh.nodes[:, 0], mesh.nodes[:, 1], mesh.nodes[:, 2]
    mask = np.zeros(3 * N, np.uint8)
    base = np.nonzero(np.abs(z) < 1.0)[0]
    for c in range(3):
        mask[3 * base + c] = 1
    mask[3 * np.nonzero((np.abs(x) < 1.0) | (np.abs(x - lx) < 1.0))[0]] = 1
    mask[3 * np.nonzero((np.abs(y) < 1.0) | (np.abs(y - ly) < 1.0))[0] + 1] = 1
    dm = geo.DofManager(N, 3)
    idx = np.nonzero(mask)[0]
    dm.set_dirichlet(idx, np.zeros(idx.size))
    mat = geo.MaxwellViscoelasticity.new(1e11, 0.25, 1e19)
    dt = 0.1 * mat.relaxation_time()
    f_ext = geo.Assembler.assemble_gravity_load(mesh, dm, 3300.0, [0.0, 0.0, -9.81], ctx)
    mesh.stress_history = geo.StressHistory(mesh.num_elements())
    mesh.stress_history.update_all(np.random.default_rng(3001).normal(0, 1e6, (mesh.num_elements(), 6)))
    csr_cg = geo.ConjugateGradient().with_tolerance(1e-8).with_max_iterations(50000)
    mixed = geo.ConjugateGradient().with_tolerance(1e-8).with_max_iterations(50000).with_precision("mixed")
    op = geo.ElasticityOperator(mesh, dm, geo.IsotropicElasticity(1e11, 0.25), None, ctx)
    u0 = np.zeros(3 * N)
    out = {}
    for name, fn in (("csr_fp64", lambda be: be.step(mesh, dm, mat, f_ext, csr_cg)),
                     ("operator_mixed", lambda be: be.step_operator(op, mesh, f_ext, mixed))):
        be = geo.BackwardEuler.new(3 * N, dt)
        fn(be)  # warm
        be.reset()
        t0 = time.perf_counter()
        u, ts = fn(be)
        t1 = time.perf_counter()
        geo.update_stresses_maxwell(mesh, dm, mat, u0, u, dt, ctx)
        t2 = time.perf_counter()
        out[name] = {"step_s": t1 - t0, "stress_update_s": t2 - t1, "iterations": ts.iterations}
        out[name + "_u"] = u
    out["step_speedup"] = out["csr_fp64"]["step_s"] / out["operator_mixed"]["step_s"]
    ua, ub = out.pop("csr_fp64_u"), out.pop("operator_mixed_u")
    out["solution_rel_l2"] = float(np.linalg.norm(ua - ub) / np.linalg.norm(ua))
    out["config"] = "48x48x24 hexes (331,776 elements, 1,383,123 DOFs), one step, host-timed"
    return out


# --------------------------------------------------------------------------- reference arm
def run_reference(args):
    n = args.size
    per_solve = []
    fp64_iters = args.ref_fp64_iters
    system = None
    for _ in range(args.warmup + args.steps):
        v, info, system = cpu_reference_sample(n, fp64_iters, args.cpu_iters, system)
        per_solve.append((v, info))
    vals = [v for v, _ in per_solve[args.warmup:]]
    info = per_solve[-1][1]
    value = statistics.median(vals)
    return {
        "metric": METRIC, "impl": "reference", "value": value, "unit": "s", "n_gpus": 1, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": 1e3 * value, "higher_is_better": False, "scaling": "weak",
        "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded ImprovedMeshGenerator cube, log-normal k)",
        "config": {"workload": f"thermal Tet10 cube {n}^3 hexes, ln k ~ N(ln 3, 0.5^2), Jacobi-PCG to rel-res 1e-8",
                   "parallelism": "serial CG (as the reference)"},
        "cpu_baseline": {"value": value, "unit": "s", "cores": 1, "kind": "port",
                         "sample": f"reference serial Jacobi-CG (C++ restatement) on the {n}^3 K_bc, "
                                   f"{args.cpu_iters} iterations per step ({info['per_iteration_s']:.3f} s/it, "
                                   f"nnz {info['nnz']}), scaled to {fp64_iters} FP64 iterations"},
        "e2e": {"value": value, "unit": "s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--size", type=int, default=128)
    ap.add_argument("--e2e-steps", type=int, default=2)
    ap.add_argument("--cpu-iters", type=int, default=5)
    ap.add_argument("--ref-fp64-iters", type=int, default=0,
                    help="FP64 iteration count to scale the reference sample by (0: measure on the GPU)")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--quick", action="store_true", help="skip FP64 / e2e / adjoint extras")
    args = ap.parse_args()
    ws, rank, local, pg = dist_setup(args)
    if args.impl == "reference":
        if rank != 0:
            return
        if args.ref_fp64_iters <= 0:
            args.ref_fp64_iters = FP64_ITERS.get(args.size, 0)
        if args.ref_fp64_iters <= 0:
            print(json.dumps({"impl": "reference", "unavailable": f"no FP64 iteration count known for size {args.size}"}))
            return
        print(json.dumps(run_reference(args)), flush=True)
        return
    line = run_ours(args, ws, rank, local, pg)
    if rank == 0:
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()


def fp64_iteration_count(n, device=0):
    """Iterations the FP64 Jacobi-PCG needs on the n^3 system (measured on the GPU)."""
    import geo_simulator_b200 as geo
    mesh, k_e, mask, vals = thermal_inputs(n)
    ctx = geo.Context.default(device)
    dm = geo.DofManager(mesh.num_nodes(), 1)
    idx = np.nonzero(mask)[0]
    dm.set_dirichlet(idx, vals[idx])
    op = geo.ThermalOperator(mesh, dm, k_e, ctx)
    f = geo.Assembler.assemble_thermal_load(mesh, dm, Q, ctx)
    _, st = op.solve(op.lift_rhs(f), geo.ConjugateGradient().with_tolerance(1e-8).with_max_iterations(20000))
    return st.iterations


if __name__ == "__main__":
    main()

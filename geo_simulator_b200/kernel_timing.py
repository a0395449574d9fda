"""Per-kernel device times of one matrix-free PCG iteration on the thermal cube.

    python -m geo_simulator_b200.kernel_timing [--size 96] [--iterations 20]
        [--nz NZ] [--precision mixed|fp64] [--physics thermal|elasticity]
    python -m geo_simulator_b200.kernel_timing --meshgen --size 128
    python -m geo_simulator_b200.kernel_timing --vtu --size 128 [--vtu-file PATH]
    python -m geo_simulator_b200.kernel_timing --csr --size 64 [--reps 2]

Builds the n^3-hex ImprovedMeshGenerator cube (1000 x 1000 x 600, ln k_e ~
N(ln 3, 0.5^2) from seed 1001, T = 1280 at z = 0 and 0 at z = 600, Q = 1e-6;
elasticity: E_e log-normal around 1e11, nu = 0.25, gravity load, roller sides),
then times `iterations` PCG iterations kernel by kernel with
geo_op_time_pcg_kernels (every launch does full work) and prints one JSON line
with the patch-kernel and node-update times and their algorithmic bytes. Used
for kernel profiles: its only launches of the PCG-mode patch kernel are the
timed ones.

With --meshgen it instead builds the same cube once on the device
(geo_mesh_generate_cube: one launch each of k_cube_vertices, k_cube_midpoints
and k_cube_conn) and prints its sizes and the mesh's algorithmic bytes.

With --csr it assembles K_bc of the cube (k = 3) on the device and runs the FP64
CSR Jacobi-PCG drop-in (geo_cg_solve, one persistent k_csr_pcg launch per solve)
to rel-res 1e-8, timed with CUDA events, and prints the iteration count and the
CSR bytes streamed per iteration.

With --vtu it builds that device mesh, attaches a seeded temperature field
(N(600, 300^2) per node, seed 9) and renders the VTU text into a device buffer
(geo_vtu_render: per section one k_item_lengths and one k_item_write launch),
timed with CUDA events, then optionally streams the same text to a file.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json

import numpy as np

LX, LY, LZ = 1000.0, 1000.0, 600.0


# qdata values per element of the affine operators: thermal G (6), elasticity J^-1 and s (10)
NQD = {1: 6, 3: 10}


def patch_pcg_bytes(E, N, s, dpn=1, zform=False):
    """Bytes one PCG-mode patch-kernel launch must move: per element its paired
    16-bit patch-local connectivity (20 B) and its qdata (6 or 10 values of s
    bytes); per DOF r, D^-1 and the previous p read, the new p and q = K p written
    (zform, the mixed thermal solver: z and the previous p read, p and q written,
    the solution read and written); the Dirichlet bitmask. (The node coordinates are
    not read: the operator stores qdata instead.)"""
    return E * (20 + NQD[dpn] * s) + N * dpn * (6 if zform else 5) * s + N / 8


def update_bytes(N, s, dpn=1, zform=False):
    """Algorithmic bytes of one node-update launch: p, q, x, r, D^-1 read, x and r
    written, Dirichlet bitmask (zform: q, z, D^-1 read, z written; p only on
    Dirichlet rows)."""
    return N * dpn * (4 if zform else 7) * s + N * dpn / 8


# Floating-point operations per element of one PCG-mode patch-kernel launch,
# counted from the kernels' own formulation (matfree.cuh, mf_kernels.cuh; an FMA
# counts two): thermal ThermalK::apply 186 (vertex sums 20, four quadrature points
# 124, outputs 42), the element's share of p.Kp 20, the fixed-point scale 10;
# elasticity ElasticK::apply 1092 (vertex sums 60, four quadrature points x 258:
# displacement gradient 78, trace 3, stress 30, its transpose back to the 30 DOFs
# 147), p.Kp 60, scale 30. Per DOF the gather forms p = D^-1 r + beta p_old (3).
PATCH_FLOPS_PER_ELEMENT = {1: 216, 3: 1182}


def patch_pcg_flops(E, N, dpn=1):
    return E * PATCH_FLOPS_PER_ELEMENT[dpn] + 3 * N * dpn


def cuda_core_peak_tflops(sm_mhz, fp64=False, sms=148):
    """Nominal CUDA-core peak of a B200 at the given SM clock: 128 FP32 (64 FP64)
    FMA lanes per SM, two flops per FMA."""
    return sms * (64 if fp64 else 128) * 2 * sm_mhz * 1e6 / 1e12


def meshgen_bytes(n_nodes, n_elem, n_vertices):
    """Algorithmic bytes of geo_mesh_generate_cube: coordinates (3 doubles per node)
    and connectivity (10 int32 per element) written once, and the int32 edge-table
    entry of every midpoint written once and read back once (the 6 reads per
    element hit L2)."""
    return 24 * n_nodes + 40 * n_elem + 8 * (n_nodes - n_vertices)


def render_device(ctx, mesh, reps=3):
    """geo_vtu_render of the mesh and its fields into a device buffer: (bytes, best
    seconds of reps by CUDA events on the context stream)."""
    import torch

    from geo_simulator_b200 import _native as N
    from geo_simulator_b200.fem import _vtu_fields
    pf, npf, keep_p = _vtu_fields(mesh.field_data)
    cf, ncf, keep_c = _vtu_fields(mesh.cell_data)
    h = mesh.handle(ctx)
    nbytes = C.c_int64()
    ctx.check(N.lib().geo_vtu_render(ctx.h, h, pf, npf, cf, ncf, None, 0, C.byref(nbytes)))
    size = int(nbytes.value)
    buf = torch.empty(size, dtype=torch.uint8, device="cuda")
    stream = torch.cuda.ExternalStream(ctx.stream_handle())
    best = None
    for _ in range(reps):
        torch.cuda.synchronize()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        ctx.check(N.lib().geo_vtu_render(ctx.h, h, pf, npf, cf, ncf, buf.data_ptr(), size, C.byref(nbytes)))
        e1.record(stream)
        torch.cuda.synchronize()
        t = e0.elapsed_time(e1) / 1e3
        best = t if best is None else min(best, t)
    return size, best


def vtu_timing(n, path=None):
    """The n^3 cube with a seeded temperature field: device render (render_device)
    and, if path is given, the streamed write to that file (wall clock)."""
    import time

    import torch

    import geo_simulator_b200 as geo
    ctx = geo.Context.default()
    dm = geo.ImprovedMeshGenerator.generate_cube_device(n, n, n, LX, LY, LZ, ctx)
    T = np.random.default_rng(9).normal(600.0, 300.0, dm.num_nodes())
    dm.field_data.add_field(geo.ScalarField("Temperature", torch.from_numpy(T).cuda()))
    size, best = render_device(ctx, dm)
    out = {"size": n, "nodes": dm.num_nodes(), "elements": dm.num_elements(), "bytes": size,
           "render_device_s": best, "render_gbs": size / best / 1e9}
    if path:
        t0 = time.perf_counter()
        geo.VtkWriter.write_vtu(dm, path, ctx)
        out["write_file_s"] = time.perf_counter() - t0
        out["write_file_gbs"] = size / out["write_file_s"] / 1e9
    return out


def build(size, physics, nz=None):
    import geo_simulator_b200 as geo
    from geo_simulator_b200.fields import lognormal_field
    mesh = geo.ImprovedMeshGenerator.generate_cube(size, size, nz or size, LX, LY, LZ)
    E, N = mesh.num_elements(), mesh.num_nodes()
    xyz = mesh.nodes
    if physics == "thermal":
        k_e = lognormal_field(1001, E, np.log(3.0), 0.5)
        z = xyz[:, 2]
        bottom = np.abs(z) < 1.0
        top = (~bottom) & (np.abs(z - LZ) < 1.0)
        d = geo.DofManager(N, 1)
        idx = np.nonzero(bottom | top)[0]
        d.set_dirichlet(idx, np.where(bottom[idx], 1280.0, 0.0))
        op = geo.ThermalOperator(mesh, d, k_e)
        f = geo.Assembler.assemble_thermal_load(mesh, d, 1e-6)
    else:
        E_e = lognormal_field(3001, E, np.log(1e11), 0.3)
        d = geo.DofManager(N, 3)
        x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
        mask = np.zeros(3 * N, np.uint8)
        mask[3 * np.nonzero(np.abs(z) < 1.0)[0] + 2] = 1
        mask[3 * np.nonzero((np.abs(x) < 1.0) | (np.abs(x - LX) < 1.0))[0]] = 1
        mask[3 * np.nonzero((np.abs(y) < 1.0) | (np.abs(y - LY) < 1.0))[0] + 1] = 1
        idx = np.nonzero(mask)[0]
        d.set_dirichlet(idx, np.zeros(idx.size))
        op = geo.ElasticityOperator(mesh, d, geo.IsotropicElasticity(1e11, 0.25), E_e)
        f = geo.Assembler.assemble_gravity_load(mesh, d, 3300.0, [0.0, 0.0, -9.81])
    return mesh, op, op.lift_rhs(f)


def csr_timing(n, reps):
    """geo_cg_solve on the assembled n^3 thermal K_bc: (JSON-ready dict)."""
    import torch

    import geo_simulator_b200 as geo
    from bench import Q, thermal_inputs
    ctx = geo.Context.default()
    mesh, _, mask, vals = thermal_inputs(n)
    dm = geo.DofManager(mesh.num_nodes(), 1)
    idx = np.nonzero(mask)[0]
    dm.set_dirichlet(idx, vals[idx])
    f = geo.Assembler.assemble_thermal_load(mesh, dm, Q, ctx)
    fd = torch.from_numpy(f).to(torch.device("cuda", torch.cuda.current_device()))
    Kb, fb = geo.Assembler.apply_dirichlet_bcs(geo.Assembler.assemble_thermal_stiffness_parallel(mesh, dm, 3.0, ctx),
                                               fd, dm, ctx)
    cg = geo.ConjugateGradient().with_tolerance(1e-8).with_max_iterations(20000)
    times, its = [], 0
    for _ in range(reps + 1):
        _, st = cg.solve(Kb, fb)
        times.append(st.solve_time)
        its = st.iterations
    t = min(times[1:]) if reps > 0 else times[0]
    nnz, rows = Kb.nnz(), Kb.rows()
    per_it = nnz * 12 + rows * 8 * 10  # CSR values + indices, and the vector streams of one iteration
    return {"size": n, "rows": rows, "nnz": nnz, "iterations": its, "solve_s": t,
            "ms_per_iteration": t / max(1, its) * 1e3, "bytes_per_iteration": per_it,
            "gbs": per_it * its / t / 1e9}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=96)
    ap.add_argument("--nz", type=int, default=None, help="hexes along z (default: --size)")
    ap.add_argument("--iterations", type=int, default=20)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--physics", default="thermal", choices=["thermal", "elasticity"])
    ap.add_argument("--meshgen", action="store_true")
    ap.add_argument("--vtu", action="store_true")
    ap.add_argument("--vtu-file", default=None)
    ap.add_argument("--csr", action="store_true")
    ap.add_argument("--reps", type=int, default=2)
    args = ap.parse_args()
    from geo_simulator_b200 import _native as N
    if args.vtu:
        print(json.dumps(vtu_timing(args.size, args.vtu_file)))
        return
    if args.csr:
        print(json.dumps(csr_timing(args.size, args.reps)))
        return
    if args.meshgen:
        import geo_simulator_b200 as geo
        n = args.size
        dm = geo.ImprovedMeshGenerator.generate_cube_device(n, n, n, LX, LY, LZ)
        nv = (n + 1) ** 3
        print(json.dumps({"size": n, "nodes": dm.num_nodes(), "elements": dm.num_elements(),
                          "bytes": meshgen_bytes(dm.num_nodes(), dm.num_elements(), nv)}))
        return
    mesh, op, fb = build(args.size, args.physics, args.nz)
    prec = N.PRECISION_MIXED if args.precision == "mixed" else N.PRECISION_FP64
    pms, ums = C.c_double(), C.c_double()
    op.ctx.check(N.lib().geo_op_time_pcg_kernels(op.h, fb.ctypes.data, prec, args.iterations,
                                                 C.byref(pms), C.byref(ums)))
    E, Nn = mesh.num_elements(), mesh.num_nodes()
    s = 4 if args.precision == "mixed" else 8
    dpn = 1 if args.physics == "thermal" else 3
    zf = args.precision == "mixed"  # the mixed solver runs the z-form
    pb, ub = patch_pcg_bytes(E, Nn, s, dpn, zf), update_bytes(Nn, s, dpn, zf)
    print(json.dumps({
        "size": args.size, "nz": args.nz or args.size, "physics": args.physics, "precision": args.precision, "elements": E, "nodes": Nn,
        "iterations": args.iterations,
        "patch_ms": pms.value, "patch_bytes": pb, "patch_gbs": pb / pms.value / 1e6,
        "update_ms": ums.value, "update_bytes": ub, "update_gbs": ub / ums.value / 1e6,
    }))


if __name__ == "__main__":
    main()

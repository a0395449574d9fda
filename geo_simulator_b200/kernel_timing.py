"""Per-kernel device times of one matrix-free PCG iteration on the thermal cube.

    python -m geo_simulator_b200.kernel_timing [--size 96] [--iterations 20]
        [--precision mixed|fp64] [--physics thermal|elasticity]
    python -m geo_simulator_b200.kernel_timing --meshgen --size 128

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
"""
from __future__ import annotations

import argparse
import ctypes as C
import json

import numpy as np

LX, LY, LZ = 1000.0, 1000.0, 600.0


def patch_pcg_bytes(E, N, s, dpn=1):
    """Algorithmic bytes of one PCG-mode patch-kernel launch: per element 10 int32
    node ids and its coefficient; per node 3 coordinates, then per DOF r, D^-1 and
    the previous p read, the new p and q = K p written; the Dirichlet bitmask."""
    return E * (10 * 4 + s) + N * 3 * s + N * dpn * 5 * s + N * dpn / 8


def update_bytes(N, s, dpn=1):
    """Algorithmic bytes of one node-update launch: p, q, x, r, D^-1 read, x and r
    written, Dirichlet bitmask."""
    return N * dpn * 7 * s + N * dpn / 8


def meshgen_bytes(n_nodes, n_elem, n_vertices):
    """Algorithmic bytes of geo_mesh_generate_cube: coordinates (3 doubles per node)
    and connectivity (10 int32 per element) written once, and the int32 edge-table
    entry of every midpoint written once and read back once (the 6 reads per
    element hit L2)."""
    return 24 * n_nodes + 40 * n_elem + 8 * (n_nodes - n_vertices)


def build(size, physics):
    import geo_simulator_b200 as geo
    from geo_simulator_b200.fields import lognormal_field
    mesh = geo.ImprovedMeshGenerator.generate_cube(size, size, size, LX, LY, LZ)
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


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--size", type=int, default=96)
    ap.add_argument("--iterations", type=int, default=20)
    ap.add_argument("--precision", default="mixed", choices=["mixed", "fp64"])
    ap.add_argument("--physics", default="thermal", choices=["thermal", "elasticity"])
    ap.add_argument("--meshgen", action="store_true")
    args = ap.parse_args()
    from geo_simulator_b200 import _native as N
    if args.meshgen:
        import geo_simulator_b200 as geo
        n = args.size
        dm = geo.ImprovedMeshGenerator.generate_cube_device(n, n, n, LX, LY, LZ)
        nv = (n + 1) ** 3
        print(json.dumps({"size": n, "nodes": dm.num_nodes(), "elements": dm.num_elements(),
                          "bytes": meshgen_bytes(dm.num_nodes(), dm.num_elements(), nv)}))
        return
    mesh, op, fb = build(args.size, args.physics)
    prec = N.PRECISION_MIXED if args.precision == "mixed" else N.PRECISION_FP64
    pms, ums = C.c_double(), C.c_double()
    op.ctx.check(N.lib().geo_op_time_pcg_kernels(op.h, fb.ctypes.data, prec, args.iterations,
                                                 C.byref(pms), C.byref(ums)))
    E, Nn = mesh.num_elements(), mesh.num_nodes()
    s = 4 if args.precision == "mixed" else 8
    dpn = 1 if args.physics == "thermal" else 3
    pb, ub = patch_pcg_bytes(E, Nn, s, dpn), update_bytes(Nn, s, dpn)
    print(json.dumps({
        "size": args.size, "physics": args.physics, "precision": args.precision, "elements": E, "nodes": Nn,
        "iterations": args.iterations,
        "patch_ms": pms.value, "patch_bytes": pb, "patch_gbs": pb / pms.value / 1e6,
        "update_ms": ums.value, "update_bytes": ub, "update_gbs": ub / ums.value / 1e6,
    }))


if __name__ == "__main__":
    main()

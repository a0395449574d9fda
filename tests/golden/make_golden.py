"""Generates tests/golden/golden.npz from the CPU oracle (oracle/), which is pinned
against the reference's known-answer tests (tests/test_oracle_pins.py).

The reference itself (Rust) cannot be built in this environment, so these
vectors come from its C++ restatement. Regenerate with:
    python tests/golden/make_golden.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402

UNIT = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0, 0, 1], [0.5, 0, 0], [0.5, 0.5, 0], [0, 0.5, 0],
                 [0, 0, 0.5], [0.5, 0, 0.5], [0, 0.5, 0.5]], dtype=np.float64)


def halfspace_bc(xyz, lx, ly):
    """elasticity_halfspace_gravity.rs:75-103: fixed base (u_z, corner u_x/u_y), roller sides."""
    n = xyz.shape[0]
    mask = np.zeros(3 * n, np.uint8)
    for i, (x, y, z) in enumerate(xyz):
        if abs(z) < 1.0:
            mask[3 * i + 2] = 1
            if abs(x) < 1.0 and abs(y) < 1.0:
                mask[3 * i] = mask[3 * i + 1] = 1
        if abs(x) < 1.0 or abs(x - lx) < 1.0:
            mask[3 * i] = 1
        if abs(y) < 1.0 or abs(y - ly) < 1.0:
            mask[3 * i + 1] = 1
    return mask, np.zeros(3 * n)


def thermal_set(prefix, n, out):
    xyz, conn = orc.generate_cube(n, n, n, 1000.0, 1000.0, 600.0)
    mask, vals = orc.thermal_bc(xyz, 600.0)
    K = orc.assemble_thermal_stiffness(xyz, conn, 3.0)
    f = orc.assemble_thermal_load(xyz, conn, 1e-6)
    Kb, fb = orc.apply_dirichlet_bcs(K, f, mask, vals)
    x, st = orc.cg_solve(Kb, fb, 1000, 1e-10)
    xl, _ = orc.lu_solve(Kb, fb)
    out.update({
        f"{prefix}_xyz": xyz, f"{prefix}_conn": conn.astype(np.int32), f"{prefix}_mask": mask,
        f"{prefix}_vals": vals, f"{prefix}_K_indptr": K.indptr, f"{prefix}_K_indices": K.indices.astype(np.int32),
        f"{prefix}_K_data": K.data, f"{prefix}_f": f, f"{prefix}_Kbc_indptr": Kb.indptr,
        f"{prefix}_Kbc_indices": Kb.indices.astype(np.int32), f"{prefix}_Kbc_data": Kb.data, f"{prefix}_fbc": fb,
        f"{prefix}_x_cg": x, f"{prefix}_cg_iterations": np.int64(st.iterations), f"{prefix}_x_lu": xl,
    })


def main():
    out = {}
    # element level (element.rs:148-163 unit Tet10, curved_element.rs:34 perturbation)
    curved = UNIT.copy()
    curved[4, 1] -= 0.1
    for tag, nodes in (("unit", UNIT), ("curved", curved)):
        out[f"{tag}_nodes"] = nodes
        out[f"{tag}_Ke"] = orc.thermal_stiffness(nodes, 2.5)
        out[f"{tag}_Me"] = orc.thermal_mass(nodes, 3300.0, 1200.0)
        out[f"{tag}_fe"] = orc.thermal_load(nodes, 6.0)
        out[f"{tag}_Ke_el"] = orc.elasticity_stiffness(nodes, 100e9, 0.25)
        out[f"{tag}_fe_grav"] = orc.gravity_load(nodes, 3000.0, [0.0, 0.0, -9.81])
    thermal_set("t2", 2, out)
    thermal_set("t6", 6, out)
    # elasticity under gravity, 2x2x2 on 100 x 100 x 50 km
    xyz, conn = orc.generate_cube(2, 2, 2, 100e3, 100e3, 50e3)
    mask, vals = halfspace_bc(xyz, 100e3, 100e3)
    K = orc.assemble_elasticity_stiffness(xyz, conn, 100e9, 0.25)
    f = orc.assemble_gravity_load(xyz, conn, 3300.0, [0.0, 0.0, -9.81])
    Kb, fb = orc.apply_dirichlet_bcs(K, f, mask, vals)
    u, st = orc.cg_solve(Kb, fb, 5000, 1e-10)
    out.update({
        "e2_xyz": xyz, "e2_conn": conn.astype(np.int32), "e2_mask": mask, "e2_K_indptr": K.indptr,
        "e2_K_indices": K.indices.astype(np.int32), "e2_K_data": K.data, "e2_f": f, "e2_Kbc_indptr": Kb.indptr,
        "e2_Kbc_indices": Kb.indices.astype(np.int32), "e2_Kbc_data": Kb.data, "e2_fbc": fb, "e2_u_cg": u,
        "e2_cg_iterations": np.int64(st.iterations),
    })
    np.savez_compressed(os.path.join(HERE, "golden.npz"), **out)
    print("wrote", os.path.join(HERE, "golden.npz"), len(out), "arrays")


if __name__ == "__main__":
    main()

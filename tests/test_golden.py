"""Golden fixtures (tests/golden/golden.npz, made by tests/golden/make_golden.py).

CPU: the oracle reproduces every fixture (it is deterministic).
GPU: the product matches them -- connectivity and CSR structure bit-exact,
element matrices and CSR values within 1e-12 of the row scale, solutions
within 1e-8 relative L2.
"""
import os

import numpy as np
import pytest

GOLD = np.load(os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "golden.npz"))


def close(a, b, rtol):
    return np.abs(np.asarray(a) - np.asarray(b)).max() <= rtol * max(np.abs(b).max(), 1e-300)


def row_err(vals, ref, indptr):
    rows = np.repeat(np.arange(indptr.size - 1), np.diff(indptr))
    scale = np.zeros(indptr.size - 1)
    np.maximum.at(scale, rows, np.abs(ref))
    return (np.abs(vals - ref) / np.maximum(scale[rows], 1e-300)).max()


# ------------------------------------------------------------------------ CPU
def test_oracle_reproduces_element_fixtures(orc):
    for tag in ("unit", "curved"):
        n = GOLD[f"{tag}_nodes"]
        assert close(orc.thermal_stiffness(n, 2.5), GOLD[f"{tag}_Ke"], 1e-14)
        assert close(orc.thermal_mass(n, 3300.0, 1200.0), GOLD[f"{tag}_Me"], 1e-14)
        assert close(orc.thermal_load(n, 6.0), GOLD[f"{tag}_fe"], 1e-14)
        assert close(orc.elasticity_stiffness(n, 100e9, 0.25), GOLD[f"{tag}_Ke_el"], 1e-14)
        assert close(orc.gravity_load(n, 3000.0, [0, 0, -9.81]), GOLD[f"{tag}_fe_grav"], 1e-14)


@pytest.mark.parametrize("prefix,n", [("t2", 2), ("t6", 6)])
def test_oracle_reproduces_thermal_fixtures(orc, prefix, n):
    xyz, conn = orc.generate_cube(n, n, n, 1000.0, 1000.0, 600.0)
    assert np.array_equal(xyz, GOLD[f"{prefix}_xyz"]) and np.array_equal(conn, GOLD[f"{prefix}_conn"])
    K = orc.assemble_thermal_stiffness(xyz, conn, 3.0)
    assert np.array_equal(K.indptr, GOLD[f"{prefix}_K_indptr"])
    assert np.array_equal(K.indices, GOLD[f"{prefix}_K_indices"])
    assert row_err(K.data, GOLD[f"{prefix}_K_data"], K.indptr) <= 1e-14
    Kb, fb = orc.apply_dirichlet_bcs(K, orc.assemble_thermal_load(xyz, conn, 1e-6), GOLD[f"{prefix}_mask"],
                                     GOLD[f"{prefix}_vals"])
    assert np.array_equal(Kb.indptr, GOLD[f"{prefix}_Kbc_indptr"])
    assert close(fb, GOLD[f"{prefix}_fbc"], 1e-14)
    x, st = orc.cg_solve(Kb, fb, 1000, 1e-10)
    assert st.iterations == int(GOLD[f"{prefix}_cg_iterations"])
    assert close(x, GOLD[f"{prefix}_x_cg"], 1e-12)


# ------------------------------------------------------------------------ GPU
def _mesh_dofs(geo, xyz, conn, mask, vals, dpn):
    mesh = geo.Mesh(xyz, conn)
    d = geo.DofManager(xyz.shape[0], dpn)
    idx = np.nonzero(mask)[0]
    d.set_dirichlet(idx, vals[idx])
    return mesh, d


@pytest.mark.gpu
def test_product_element_fixtures(geo):
    for tag in ("unit", "curved"):
        n = GOLD[f"{tag}_nodes"]
        mesh = geo.Mesh(n, np.arange(10, dtype=np.int32).reshape(1, 10))
        assert close(geo.ElementMatrix.thermal_stiffness(mesh, 2.5)[0], GOLD[f"{tag}_Ke"], 1e-12)
        assert close(geo.ElementMatrix.thermal_mass(mesh, 3300.0, 1200.0)[0], GOLD[f"{tag}_Me"], 1e-12)
        assert close(geo.ElementMatrix.thermal_load(mesh, 6.0)[0], GOLD[f"{tag}_fe"], 1e-12)
        mat = geo.IsotropicElasticity(100e9, 0.25)
        assert close(geo.ElasticityElement.stiffness_matrix(mesh, mat)[0], GOLD[f"{tag}_Ke_el"], 1e-12)
        assert close(geo.BodyForce.gravity_load(mesh, 3000.0, [0, 0, -9.81])[0], GOLD[f"{tag}_fe_grav"], 1e-12)


@pytest.mark.gpu
@pytest.mark.parametrize("prefix,n", [("t2", 2), ("t6", 6)])
def test_product_thermal_fixtures(geo, prefix, n):
    m = geo.ImprovedMeshGenerator.generate_cube(n, n, n, 1000.0, 1000.0, 600.0)
    assert np.array_equal(m.nodes, GOLD[f"{prefix}_xyz"]) and np.array_equal(m.elements, GOLD[f"{prefix}_conn"])
    mesh, d = _mesh_dofs(geo, m.nodes, m.elements, GOLD[f"{prefix}_mask"], GOLD[f"{prefix}_vals"], 1)
    K = geo.Assembler.assemble_thermal_stiffness_parallel(mesh, d, 3.0)
    ip, ix, data = K.to_host()
    assert np.array_equal(ip, GOLD[f"{prefix}_K_indptr"]) and np.array_equal(ix, GOLD[f"{prefix}_K_indices"])
    assert row_err(data, GOLD[f"{prefix}_K_data"], ip) <= 1e-12
    f = geo.Assembler.assemble_thermal_load(mesh, d, 1e-6)
    assert close(f, GOLD[f"{prefix}_f"], 1e-12)
    Kb, fb = geo.Assembler.apply_dirichlet_bcs(K, f, d)
    ip, ix, data = Kb.to_host()
    assert np.array_equal(ip, GOLD[f"{prefix}_Kbc_indptr"]) and np.array_equal(ix, GOLD[f"{prefix}_Kbc_indices"])
    assert row_err(data, GOLD[f"{prefix}_Kbc_data"], ip) <= 1e-12
    assert close(fb, GOLD[f"{prefix}_fbc"], 1e-12)
    x, st = geo.ConjugateGradient().with_tolerance(1e-10).solve(Kb, fb)
    assert st.iterations == int(GOLD[f"{prefix}_cg_iterations"])
    xg = GOLD[f"{prefix}_x_cg"]
    assert np.linalg.norm(x - xg) / np.linalg.norm(xg) <= 1e-8
    xl = GOLD[f"{prefix}_x_lu"]
    assert np.linalg.norm(x - xl) / np.linalg.norm(xl) <= 1e-8
    op = geo.ThermalOperator(mesh, d, 3.0)
    for prec in ("fp64", "mixed"):
        xm, sm = op.solve(GOLD[f"{prefix}_fbc"], geo.ConjugateGradient().with_tolerance(1e-10).with_precision(prec))
        assert sm.converged and np.linalg.norm(xm - xl) / np.linalg.norm(xl) <= 1e-8


@pytest.mark.gpu
def test_product_elasticity_fixture(geo):
    xyz, conn, mask = GOLD["e2_xyz"], GOLD["e2_conn"], GOLD["e2_mask"]
    mesh, d = _mesh_dofs(geo, xyz, conn, mask, np.zeros(mask.size), 3)
    mat = geo.IsotropicElasticity(100e9, 0.25)
    K = geo.Assembler.assemble_elasticity_stiffness_parallel(mesh, d, mat)
    ip, ix, data = K.to_host()
    assert np.array_equal(ip, GOLD["e2_K_indptr"]) and np.array_equal(ix, GOLD["e2_K_indices"])
    assert row_err(data, GOLD["e2_K_data"], ip) <= 1e-12
    f = geo.Assembler.assemble_gravity_load(mesh, d, 3300.0, [0.0, 0.0, -9.81])
    assert close(f, GOLD["e2_f"], 1e-12)
    Kb, fb = geo.Assembler.apply_dirichlet_bcs(K, f, d)
    ip, ix, data = Kb.to_host()
    assert np.array_equal(ip, GOLD["e2_Kbc_indptr"]) and np.array_equal(ix, GOLD["e2_Kbc_indices"])
    assert row_err(data, GOLD["e2_Kbc_data"], ip) <= 1e-12
    assert close(fb, GOLD["e2_fbc"], 1e-12)
    u, st = geo.ConjugateGradient().with_max_iterations(5000).with_tolerance(1e-10).solve(Kb, fb)
    # same loop; the SpMV sums in a different order, which can move the stopping
    # point of this stiffer system by an iteration
    assert st.converged and abs(st.iterations - int(GOLD["e2_cg_iterations"])) <= 2
    ug = GOLD["e2_u_cg"]
    assert np.linalg.norm(u - ug) / np.linalg.norm(ug) <= 1e-8

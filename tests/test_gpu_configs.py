"""Parity at the benchmark configurations' own sizes (not only toy meshes).

* 64^3 thermal cube (1,572,864 elements, 2,146,689 DOFs, k = 3): connectivity
  bit-exact against the oracle's generate_cube; K_e of every element within
  1e-12 of element.rs:23-61 restated; the CSR of assemble_thermal_stiffness_parallel
  (assembly.rs:69-117) and of apply_dirichlet_bcs (:168-230) bit-exact in structure
  (nnz 60,859,905 and 59,755,513) and within 1e-12 (row scale) in value, with f_bc.
* 48x48x32 inversion box (442,368 elements, 611,585 DOFs, ln k ~ N(ln 3, 0.3^2),
  seed 2001): the mixed-precision adjoint gradient dJ/d(ln k_e) of
  J = 1/2 sum over 1000 seeded free nodes (seed 2003) of (T - T_hat)^2, T_hat from a
  forward solve with ln k + 0.1 N(0, 1) (seed 2002), against FP64 central finite
  differences (h = 1e-6) on 20 seeded elements (seed 2004), 1e-5 relative, no floor.
* 48x48x24 elasticity half-space (331,776 elements, 1,383,123 DOFs, ln E ~
  N(ln 1e11, 0.3^2), seed 3001, fixed base, roller sides): dJ/d(ln E_e) of the
  surface misfit 1/2 sum over 500 seeded top nodes (seed 3002) of (u_z - u_hat_z)^2,
  u_hat from ln E + 0.1 N(0, 1) (seed 3003), on 10 seeded elements (seed 3004).
* The accuracy contract of the mixed solver on a 32^3 log-normal cube (sigma 0.5,
  seed 1001): stopped at rel-res 1e-11 like the FP64 solver, the two solutions
  agree to 1e-8 relative L2; and mixed solves are bit-reproducible.

Finite differences. J(ln k_e +- h) needs the forward state of the perturbed
coefficients. It is computed by residual correction from the converged state u
(FP64 solve to rel-res 1e-13): with r0 = f_bc - K_bc u (one FP64 apply, shared by
both signs) and dK = (e^{+-h} - 1) K_e (K_e linear in its coefficient, K_e from the
oracle), the perturbed system's residual at u is r0 - dK u on the free rows, and
u' = u + K'^{-1}(r0 - dK u) with an FP64 solve of K' (rel-res 1e-13 on that small
right-hand side). J+ - J- = 1/2 sum (d+ - d-)(2(u - T_hat) + d+ + d-) avoids the
cancellation of J+ - J-. The perturbed states are then exact to far below the
1e-5 check, for every element, so the check needs no floor on small gradients.
"""
import numpy as np
import pytest

from geo_simulator_b200.fields import choice_distinct, lognormal_field

pytestmark = pytest.mark.gpu

RTOL = 1e-12
L3 = (1000.0, 1000.0, 600.0)


def rel(a, b):
    return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(b), 1e-300))


def row_scaled_err(gpu_vals, orc_vals, indptr):
    """max |gpu - oracle| / max |row of the oracle| over all entries (no empty rows)."""
    scale = np.maximum.reduceat(np.abs(orc_vals), indptr[:-1])
    rows = np.repeat(np.arange(indptr.size - 1), np.diff(indptr))
    return float((np.abs(gpu_vals - orc_vals) / np.maximum(scale[rows], 1e-300)).max())


def dof_mgr(geo, n, mask, vals, dpn=1):
    d = geo.DofManager(n, dpn)
    idx = np.nonzero(mask)[0]
    d.set_dirichlet(idx, vals[idx])
    return d


def test_c2_connectivity_element_matrices_and_csr_at_size(orc, geo):
    n = 64
    xyz, conn = orc.generate_cube(n, n, n, *L3)
    mesh = geo.ImprovedMeshGenerator.generate_cube(n, n, n, *L3)
    assert conn.shape[0] == 1_572_864 and xyz.shape[0] == 2_146_689
    assert np.array_equal(mesh.elements, conn) and np.array_equal(mesh.nodes.view(np.uint64), xyz.view(np.uint64))
    # K_e of every element
    Ke = geo.ElementMatrix.thermal_stiffness(mesh, 3.0)
    Ko = orc.thermal_stiffness_all(xyz, conn, 3.0)
    worst = 0.0
    for a in range(0, conn.shape[0], 1 << 18):
        g, o = Ke[a:a + (1 << 18)], Ko[a:a + (1 << 18)]
        worst = max(worst, float((np.abs(g - o).max(axis=(1, 2)) / np.abs(o).max(axis=(1, 2))).max()))
    assert worst <= RTOL, worst
    del Ke, Ko
    # CSR K and K_bc, f and f_bc
    mask, vals = orc.thermal_bc(xyz, L3[2])
    dm = dof_mgr(geo, xyz.shape[0], mask, vals)
    K = geo.Assembler.assemble_thermal_stiffness_parallel(mesh, dm, 3.0)
    K_o = orc.assemble_thermal_stiffness(xyz, conn, 3.0)  # rayon element loop + triplet merge, restated
    ip, ix, d = K.to_host()
    assert K.nnz() == 60_859_905 == K_o.nnz
    assert np.array_equal(ip, K_o.indptr) and np.array_equal(ix.astype(np.int64), K_o.indices)
    assert row_scaled_err(d, K_o.data, ip) <= RTOL
    f = geo.Assembler.assemble_thermal_load(mesh, dm, 1e-6)
    f_o = orc.assemble_thermal_load(xyz, conn, 1e-6)
    assert np.abs(f - f_o).max() <= RTOL * np.abs(f_o).max()
    Kb, fb = geo.Assembler.apply_dirichlet_bcs(K, f, dm)
    Kb_o, fb_o = orc.apply_dirichlet_bcs(K_o, f_o, mask, vals)
    ip, ix, d = Kb.to_host()
    assert Kb.nnz() == 59_755_513 == Kb_o.nnz
    assert np.array_equal(ip, Kb_o.indptr) and np.array_equal(ix.astype(np.int64), Kb_o.indices)
    assert row_scaled_err(d, Kb_o.data, ip) <= RTOL
    assert np.abs(fb - fb_o).max() <= RTOL * np.abs(fb_o).max()


def _perturbed_states(op, u_full, r0, coef, e, h, Ke_e, dofs_e, dir_mask, solver, bnorm):
    """State differences d+- = u(coef_e e^{+-h}) - u by residual correction (module doc).
    The correction's right-hand side is tiny; it is solved scaled to the forward
    right-hand side's norm bnorm (the system is linear), so that the CG's absolute
    thresholds (breakdown at |p.Ap| < 1e-30, iterative.rs:85) see the magnitudes
    of a forward solve."""
    out = []
    for sgn in (1.0, -1.0):
        c = coef.copy()
        c[e] = coef[e] * np.exp(sgn * h)
        op.set_coefficients(c)
        r = r0.copy()
        r[dofs_e] -= np.expm1(sgn * h) * (Ke_e @ u_full[dofs_e])
        r[dir_mask == 1] = 0.0
        sc = bnorm / np.linalg.norm(r)
        d, st = op.solve(r * sc, solver)
        assert st.converged, st
        out.append(d / sc)
    op.set_coefficients(coef)
    return out


def _fd(dp, dm, u, that, obs, h):
    return 0.5 * np.sum((dp[obs] - dm[obs]) * (2.0 * (u[obs] - that[obs]) + dp[obs] + dm[obs])) / (2.0 * h)


def test_c4_adjoint_gradient_vs_central_differences_at_size(orc, geo):
    nx, ny, nz = 48, 48, 32
    xyz, conn = orc.generate_cube(nx, ny, nz, *L3)
    E = conn.shape[0]
    assert E == 442_368 and xyz.shape[0] == 611_585
    mask, vals = orc.thermal_bc(xyz, L3[2])
    mesh = geo.Mesh(xyz, conn.astype(np.int32))
    dm = dof_mgr(geo, xyz.shape[0], mask, vals)
    lnk = lognormal_field(2001, E, np.log(3.0), 0.3, log=True)
    k = np.exp(lnk)
    op = geo.ThermalOperator(mesh, dm, k)
    f = geo.Assembler.assemble_thermal_load(mesh, dm, 1e-6)
    fp64 = geo.ConjugateGradient().with_max_iterations(50000).with_tolerance(1e-13).with_abs_tolerance(0.0)
    op.set_coefficients(np.exp(lnk + 0.1 * lognormal_field(2002, E, 0.0, 1.0, log=True)))
    that, st = op.forward(f, fp64)
    assert st.converged
    op.set_coefficients(k)
    u, st = op.forward(f, fp64)
    assert st.converged
    free = np.nonzero(mask == 0)[0]
    obs = free[choice_distinct(2003, free.size, 1000)]
    dJ = np.zeros_like(u)
    dJ[obs] = u[obs] - that[obs]
    mixed = geo.ConjugateGradient().with_max_iterations(50000).with_tolerance(1e-12).with_precision("mixed")
    grad, sa = op.vjp(dJ, u=u, solver=mixed)
    assert sa.converged
    u_full = np.where(mask == 1, vals, u)
    fb = op.lift_rhs(f)
    r0 = fb - op.apply(u_full)
    h = 1e-6
    for e in choice_distinct(2004, E, 20):
        Ke_e = orc.thermal_stiffness(xyz[conn[e]], k[e])
        dp, dmn = _perturbed_states(op, u_full, r0, k, e, h, Ke_e, conn[e], mask, fp64, np.linalg.norm(fb))
        fd = _fd(dp, dmn, u, that, obs, h)
        assert abs(grad[e] - fd) <= 1e-5 * abs(fd), (int(e), grad[e], fd)


def test_c5_elasticity_adjoint_gradient_vs_central_differences_at_size(orc, geo):
    nx, ny, nz, lx, ly, lz = 48, 48, 24, 100e3, 100e3, 50e3
    xyz, conn = orc.generate_cube(nx, ny, nz, lx, ly, lz)
    E = conn.shape[0]
    nn = xyz.shape[0]
    assert E == 331_776 and nn == 461_041
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    mask = np.zeros(3 * nn, np.uint8)
    base = np.nonzero(np.abs(z) < 1.0)[0]
    for c in range(3):
        mask[3 * base + c] = 1
    mask[3 * np.nonzero((np.abs(x) < 1.0) | (np.abs(x - lx) < 1.0))[0]] = 1
    mask[3 * np.nonzero((np.abs(y) < 1.0) | (np.abs(y - ly) < 1.0))[0] + 1] = 1
    vals = np.zeros(3 * nn)
    mesh = geo.Mesh(xyz, conn.astype(np.int32))
    dm = dof_mgr(geo, nn, mask, vals, 3)
    lnE = lognormal_field(3001, E, np.log(1e11), 0.3, log=True)
    Ee = np.exp(lnE)
    op = geo.ElasticityOperator(mesh, dm, geo.IsotropicElasticity(1e11, 0.25), Ee)
    f = geo.Assembler.assemble_gravity_load(mesh, dm, 3300.0, [0.0, 0.0, -9.81])
    fp64 = geo.ConjugateGradient().with_max_iterations(100000).with_tolerance(1e-13).with_abs_tolerance(0.0)
    op.set_coefficients(np.exp(lnE + 0.1 * lognormal_field(3003, E, 0.0, 1.0, log=True)))
    uhat, st = op.forward(f, fp64)
    assert st.converged
    op.set_coefficients(Ee)
    u, st = op.forward(f, fp64)
    assert st.converged
    top = np.nonzero(np.abs(z - lz) < 1.0)[0]
    obs = 3 * top[choice_distinct(3002, top.size, 500)] + 2
    dJ = np.zeros_like(u)
    dJ[obs] = u[obs] - uhat[obs]
    mixed = geo.ConjugateGradient().with_max_iterations(100000).with_tolerance(1e-12).with_precision("mixed")
    grad, sa = op.vjp(dJ, u=u, solver=mixed)
    assert sa.converged
    u_full = np.where(mask == 1, vals, u)
    fb = op.lift_rhs(f)
    r0 = fb - op.apply(u_full)
    h = 1e-6
    for e in choice_distinct(3004, E, 10):
        Ke_e = orc.elasticity_stiffness(xyz[conn[e]], Ee[e], 0.25)
        dofs = (3 * conn[e][:, None] + np.arange(3)).ravel()
        dp, dmn = _perturbed_states(op, u_full, r0, Ee, e, h, Ke_e, dofs, mask, fp64, np.linalg.norm(fb))
        fd = _fd(dp, dmn, u, uhat, obs, h)
        assert abs(grad[e] - fd) <= 1e-5 * abs(fd), (int(e), grad[e], fd)


@pytest.fixture(scope="module")
def cube32(geo):
    n = 32
    mesh = geo.ImprovedMeshGenerator.generate_cube(n, n, n, *L3)
    k = lognormal_field(1001, mesh.num_elements(), np.log(3.0), 0.5)
    z = mesh.nodes[:, 2]
    bottom = np.abs(z) < 1.0
    mask = (bottom | (np.abs(z - L3[2]) < 1.0)).astype(np.uint8)
    vals = np.where(bottom, 1280.0, 0.0)
    dm = dof_mgr(geo, mesh.num_nodes(), mask, vals)
    op = geo.ThermalOperator(mesh, dm, k)
    f = geo.Assembler.assemble_thermal_load(mesh, dm, 1e-6)
    return op, op.lift_rhs(f), f


def test_mixed_agrees_with_fp64_under_the_contract_rule(cube32, geo):
    """Both solvers stopped at rel-res 1e-11 (the benchmark's stopping rule):
    mixed and FP64 solutions agree to 1e-8 relative L2, and both sit within 1e-8 of
    a solve converged to rel-res 1e-13."""
    op, fb, _ = cube32
    cg = lambda t: geo.ConjugateGradient().with_max_iterations(50000).with_tolerance(t)
    xm, sm = op.solve(fb, cg(1e-11).with_precision("mixed"))
    x64, s64 = op.solve(fb, cg(1e-11))
    xc, sc = op.solve(fb, cg(1e-13))
    assert sm.converged and s64.converged and sc.converged
    assert np.linalg.norm(fb - op.apply(xm)) / np.linalg.norm(fb) < 1e-11
    assert rel(xm, x64) <= 1e-8
    assert rel(xm, xc) <= 1e-8 and rel(x64, xc) <= 1e-8


def test_mixed_solve_and_forward_bit_reproducible(cube32, geo):
    """Halo mode everywhere (PCG, FP64 refresh apply, lift): no global atomics, so two
    mixed solves of one operator give identical iterates and iteration counts."""
    op, fb, f = cube32
    s = geo.ConjugateGradient().with_max_iterations(50000).with_tolerance(1e-10).with_precision("mixed")
    xa, sa = op.solve(fb, s)
    xb, sb = op.solve(fb, s)
    assert sa.iterations == sb.iterations and sa.fp64_residual_updates == sb.fp64_residual_updates
    assert np.array_equal(xa, xb)
    ua, _ = op.forward(f, s)
    ub, _ = op.forward(f, s)
    assert np.array_equal(ua, ub)
    x = np.random.default_rng(1).standard_normal(fb.size)
    assert np.array_equal(op.apply(x), op.apply(x))
    assert np.array_equal(op.lift_rhs(f), op.lift_rhs(f))

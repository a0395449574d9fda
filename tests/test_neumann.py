"""Neumann (flux) boundary conditions: Tet10Face::from_element_face / area /
integrate_flux (fem/boundary.rs:89-266), Assembler::find_boundary_faces
(assembly.rs:287-309) and Assembler::apply_neumann_bcs (assembly.rs:248-274).

CPU: the oracle against the reference's own tests (boundary.rs:272-310) and the
integral identities; the Python mirror's face table and BC container.
GPU: face fluxes, areas, boundary-face detection and the assembled load against
the oracle, and the analytic 1D profile with a prescribed flux."""
import numpy as np
import pytest

TRI = np.array([[0, 0, 0], [1, 0, 0], [0, 1, 0], [0.5, 0, 0], [0.5, 0.5, 0], [0, 0.5, 0]], float)


# ------------------------------------------------------------------------ CPU
def test_oracle_face_extraction_and_area(orc):
    """boundary.rs:289-297 (face 3 of 0..9 is [0,1,2,4,5,6]) and :299-323 (area 0.5)."""
    assert list(orc.face_nodes(np.arange(10), 3)) == [0, 1, 2, 4, 5, 6]
    assert list(orc.face_nodes(np.arange(10), 0)) == [1, 2, 3, 5, 9, 8]
    assert abs(orc.face_area(TRI) - 0.5) < 1e-10


def test_oracle_flux_identities(orc):
    # constant flux: sum of nodal loads = flux * area; P2 triangle: vertex loads 0, midpoints A/3
    f = orc.face_flux(TRI, 100.0)
    assert abs(f.sum() - 50.0) < 1e-12
    assert np.abs(f[:3]).max() < 1e-12 and np.allclose(f[3:], 50.0 / 3, rtol=1e-14)
    # a tilted, curved face: sum = flux * area still
    c = TRI.copy() * [2.0, 3.0, 1.0]
    c[:, 2] = 0.3 * c[:, 0] - 0.2 * c[:, 1]
    c[4] += [0.05, -0.02, 0.07]
    f = orc.face_flux(c, 2.5)
    assert abs(f.sum() - 2.5 * orc.face_area(c)) < 1e-12 * abs(f).sum()


def test_mirror_face_table_and_container(geo, orc):
    for lf in range(4):
        assert np.array_equal(geo.Tet10Face.from_element_face(np.arange(10) * 7, lf).nodes,
                              orc.face_nodes(np.arange(10) * 7, lf))
    with pytest.raises(geo.GeoError):
        geo.Tet10Face.from_element_face(np.arange(10), 4)
    bcs = geo.BoundaryConditions.new()
    face = geo.BoundaryFace(0, 3)
    bcs.add_neumann(face, 100.0)
    assert bcs.num_neumann_bcs() == 1 and bcs.get_neumann(face).flux == 100.0  # boundary.rs:272-287


def test_oracle_find_faces_on_cube(orc):
    xyz, conn = orc.generate_cube(3, 2, 2, 1000.0, 1000.0, 600.0)
    faces = orc.find_boundary_faces(conn, np.abs(xyz[:, 2] - 600.0) < 1.0)
    assert faces.shape == (3 * 2 * 2, 2)  # two triangles per top hex face
    area = sum(orc.face_area(xyz[orc.face_nodes(conn[e], lf)]) for e, lf in faces)
    assert abs(area - 1000.0 * 1000.0) < 1e-6


# ------------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_face_flux_and_area_match_oracle(orc, geo):
    xyz, conn = orc.generate_cube(2, 2, 2, 1000.0, 800.0, 600.0)
    rng = np.random.default_rng(7)
    xyz = xyz + rng.uniform(-20, 20, xyz.shape) * (np.arange(xyz.shape[0]) >= 27)[:, None]  # curved faces
    mesh = geo.Mesh(xyz, conn.astype(np.int32))
    faces = np.array([[e, lf] for e in range(conn.shape[0]) for lf in range(4)], np.int32)
    flux = rng.uniform(-5, 5, faces.shape[0])
    fe = geo.Tet10Face.integrate_flux_faces(mesh, faces, flux)
    area = geo.Tet10Face.area_faces(mesh, faces)
    for k, (e, lf) in enumerate(faces):
        c = xyz[orc.face_nodes(conn[e], lf)]
        ref = orc.face_flux(c, flux[k])
        assert np.abs(fe[k] - ref).max() <= 1e-12 * np.abs(ref).max()
        assert abs(area[k] - orc.face_area(c)) <= 1e-12 * area[k]
    with pytest.raises(geo.GeoError):
        geo.Tet10Face.integrate_flux_faces(mesh, np.array([[0, 4]], np.int32), 1.0)


@pytest.mark.gpu
def test_find_faces_and_apply_neumann_match_oracle(orc, geo):
    xyz, conn = orc.generate_cube(4, 3, 3, 1000.0, 1000.0, 600.0)
    mesh = geo.Mesh(xyz, conn.astype(np.int32))
    for cond in (lambda p: np.abs(p[:, 2] - 600.0) < 1.0, lambda p: np.abs(p[:, 0]) < 1.0,
                 lambda p: (np.abs(p[:, 1] - 1000.0) < 1.0) & (p[:, 2] > 150.0)):
        faces = geo.Assembler.find_boundary_faces(mesh, cond)
        ref = orc.find_boundary_faces(conn, cond(xyz))
        assert np.array_equal(faces, ref.astype(np.int32))
    faces = geo.Assembler.find_boundary_faces(mesh, lambda p: np.abs(p[:, 2] - 600.0) < 1.0)
    flux = np.random.default_rng(8).uniform(0.5, 2.0, faces.shape[0])
    f0 = np.random.default_rng(9).standard_normal(xyz.shape[0])
    f = geo.Assembler.apply_neumann_bcs(mesh, f0.copy(), (faces, flux))
    fo = orc.apply_neumann_bcs(xyz, conn, faces, flux, f0)
    assert np.abs(f - fo).max() <= 1e-12 * np.abs(fo).max()
    bcs = geo.BoundaryConditions()
    for (e, lf), q in zip(faces, flux):
        bcs.add_neumann(geo.BoundaryFace(int(e), int(lf)), q)
    f2 = geo.Assembler.apply_neumann_bcs(mesh, f0.copy(), bcs)
    assert np.array_equal(f2, f)  # deterministic
    import torch
    fd = torch.from_numpy(f0.copy()).cuda()
    geo.Assembler.apply_neumann_bcs(mesh, fd, (faces, flux))
    assert np.abs(fd.cpu().numpy() - fo).max() <= 1e-12 * np.abs(fo).max()


@pytest.mark.gpu
@pytest.mark.parametrize("n", [2, 4])
def test_flux_profile_is_exact(geo, n):
    """-k T'' = Q, T(0) = T0, k T'(L) = q: T = T0 + (Q L + q) z / k - Q z^2 / (2 k), exact for P2."""
    lz, k, Q, T0, q = 600.0, 3.0, 1e-6, 1280.0, 0.02
    mesh = geo.ImprovedMeshGenerator.generate_cube(n, n, n, 1000.0, 1000.0, lz)
    z = mesh.nodes[:, 2]
    d = geo.DofManager(mesh.num_nodes(), 1)
    bottom = np.nonzero(np.abs(z) < 1.0)[0]
    d.set_dirichlet(bottom, np.full(bottom.size, T0))
    K = geo.Assembler.assemble_thermal_stiffness_parallel(mesh, d, k)
    f = geo.Assembler.assemble_thermal_load(mesh, d, Q)
    top = geo.Assembler.find_boundary_faces(mesh, lambda p: np.abs(p[:, 2] - lz) < 1.0)
    geo.Assembler.apply_neumann_bcs(mesh, f, (top, q))
    Kb, fb = geo.Assembler.apply_dirichlet_bcs(K, f, d)
    T, st = geo.ConjugateGradient().with_max_iterations(2000).with_tolerance(1e-12).solve(Kb, fb)
    exact = T0 + (Q * lz + q) * z / k - Q * z * z / (2 * k)
    assert st.converged and np.abs(T - exact).max() <= 1e-6 * np.abs(exact).max()

"""VTU output: VtkWriter::write_vtu (mesh/vtk_writer.rs:104-265), with every f64
printed by Rust's `{}` and every index by `{}` for usize.

CPU: the oracle's Rust Display of f64 against Python's repr (David Gay's
shortest round-trip conversion, an independent implementation) re-laid out in
Rust's positional style, on random bit patterns, every power of two and its
neighbours, subnormals and specials; known answers of Rust's Display; the
oracle's file against a Python restatement of the writer and the committed
golden file.
GPU: the device text against the oracle and the golden file byte for byte, on
bit-pattern fields covering every class of double; every sink (host buffer,
device buffer, file) gives the same bytes; streaming across many chunks (64^3)
round-trips every coordinate and index; capacity errors."""
import math
import os

import numpy as np
import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
GOLDEN = os.path.join(HERE, "golden", "vtu_2x1x1.vtu")


def rust_display_from_repr(v: float) -> str:
    """Rust `{}` of an f64 from Python's repr digits (shortest round trip)."""
    v = float(v)
    if math.isnan(v):
        return "NaN"
    sign = "-" if math.copysign(1.0, v) < 0 else ""
    a = abs(v)
    if math.isinf(a):
        return sign + "inf"
    if a == 0:
        return sign + "0"
    r = repr(a)
    m, e = (r.split("e") + ["0"])[:2]
    e = int(e)
    ip, fp = (m.split(".") + [""])[:2]
    alld = ip + fp
    lead = len(alld) - len(alld.lstrip("0"))
    digits = alld[lead:].rstrip("0")
    x = e + len(ip) - lead
    n = len(digits)
    if x <= 0:
        return sign + "0." + "0" * (-x) + digits
    if x < n:
        return sign + digits[:x] + "." + digits[x:]
    return sign + digits + "0" * (x - n)


def sample_doubles(n_random, seed=3):
    rng = np.random.default_rng(seed)
    bits = rng.integers(0, 2**64, n_random, dtype=np.uint64)
    vals = list(bits.view(np.float64))
    for e in range(-1074, 1024):
        x = 2.0**e
        vals += [x, math.nextafter(x, 0.0), math.nextafter(x, math.inf), -x]
    vals += [c * 5e-324 for c in range(1, 400)]
    vals += [0.0, -0.0, math.inf, -math.inf, math.nan, 0.1 + 0.2, 1e21, 1e-7, 7.8125, 2.0**53 + 2,
             1.7976931348623157e308, 2.2250738585072014e-308]
    vals += list(rng.uniform(-2000, 2000, 2000)) + list(np.round(rng.uniform(0, 1e6, 2000)) / 128)
    return np.array(vals, np.float64)


def python_write_vtu(xyz, conn, pf, cf) -> bytes:
    """A second restatement of vtk_writer.rs:104-265 (Python, repr-based digits)."""
    f = rust_display_from_repr
    out = ['<?xml version="1.0"?>\n',
           '<VTKFile type="UnstructuredGrid" version="1.0" byte_order="LittleEndian">\n',
           "  <UnstructuredGrid>\n",
           f'    <Piece NumberOfPoints="{xyz.shape[0]}" NumberOfCells="{conn.shape[0]}">\n',
           "      <Points>\n",
           '        <DataArray type="Float64" NumberOfComponents="3" format="ascii">\n']
    out += [f"          {f(p[0])} {f(p[1])} {f(p[2])}\n" for p in xyz]
    out += ["        </DataArray>\n", "      </Points>\n", "      <Cells>\n",
            '        <DataArray type="Int32" Name="connectivity" format="ascii">\n', "          "]
    out += [f"{int(i)} " for i in conn.reshape(-1)]
    out += ["\n        </DataArray>\n", '        <DataArray type="Int32" Name="offsets" format="ascii">\n',
            "          "]
    out += [f"{10 * (i + 1)} " for i in range(conn.shape[0])]
    out += ["\n        </DataArray>\n", '        <DataArray type="UInt8" Name="types" format="ascii">\n',
            "          "]
    out += ["24 "] * conn.shape[0]
    out += ["\n        </DataArray>\n", "      </Cells>\n"]
    for tag, fields in (("PointData", pf), ("CellData", cf)):
        if not fields:
            continue
        out.append(f"      <{tag}>\n")
        for vec in (False, True):
            for name, data, comps in fields:
                if (comps == 3) != vec:
                    continue
                extra = ' NumberOfComponents="3"' if vec else ""
                out.append(f'        <DataArray type="Float64" Name="{name}"{extra} format="ascii">\n          ')
                out += [f(v) + " " for v in np.asarray(data, np.float64).reshape(-1)]
                out.append("\n        </DataArray>\n")
        out.append(f"      </{tag}>\n")
    out += ["    </Piece>\n", "  </UnstructuredGrid>\n", "</VTKFile>\n"]
    return "".join(out).encode()


NODAL_NAMES = ["PlasticStrain", "Stress_II", "StrainRate_II", "Pressure", "Viscosity", "IsYielding",
               "YieldStress", "PlasticViscosity", "SoftenedCohesion"]


def python_write_vtk(xyz, conn, pf, cf) -> bytes:
    """A second restatement of VtkWriter::write (vtk_writer.rs:13-101)."""
    f = rust_display_from_repr
    out = ["# vtk DataFile Version 3.0\n", "Tet10 Mesh generated by geo_simulator\n", "ASCII\n",
           "DATASET UNSTRUCTURED_GRID\n", f"POINTS {xyz.shape[0]} double\n"]
    out += [f"{f(p[0])} {f(p[1])} {f(p[2])}\n" for p in xyz]
    out.append(f"\nCELLS {conn.shape[0]} {11 * conn.shape[0]}\n")
    out += ["10" + "".join(f" {int(i)}" for i in row) + "\n" for row in conn]
    out.append(f"\nCELL_TYPES {conn.shape[0]}\n")
    out += ["24\n"] * conn.shape[0]
    for tag, count, fields in (("POINT_DATA", xyz.shape[0], pf), ("CELL_DATA", conn.shape[0], cf)):
        if not fields:
            continue
        out.append(f"\n{tag} {count}\n")
        for vec in (False, True):
            for name, data, comps in fields:
                if (comps == 3) != vec:
                    continue
                d = np.asarray(data, np.float64).reshape(-1, comps)
                if vec:
                    out.append(f"VECTORS {name} double\n")
                    out += [f"{f(v[0])} {f(v[1])} {f(v[2])}\n" for v in d]
                else:
                    out.append(f"SCALARS {name} double 1\nLOOKUP_TABLE default\n")
                    out += [f"{f(v[0])}\n" for v in d]
    return "".join(out).encode()


def python_write_vtu_nodal(xyz, conn, pf, cf) -> bytes:
    """A second restatement of VtkWriter::write_nodal_vtu (vtk_writer.rs:531-789)."""
    f = rust_display_from_repr
    head = python_write_vtu(xyz, conn, [], []).decode()
    head = head[:head.index("    </Piece>")]
    n = xyz.shape[0]
    cells = {name: np.asarray(data, np.float64) for name, data, comps in cf if comps == 1}
    nodal = {k: np.zeros(n) for k in NODAL_NAMES}
    count = np.zeros(n, np.int64)
    for k in NODAL_NAMES:
        if k not in cells:
            continue
        for e in range(conn.shape[0]):  # element order, as the reference
            for node in conn[e]:
                nodal[k][node] += cells[k][e]
                if k == "PlasticStrain":
                    count[node] += 1
    for k in NODAL_NAMES:
        nodal[k] = np.where(count > 0, nodal[k] / np.maximum(count, 1), nodal[k])
    out = [head, "      <PointData>\n"]
    for name, data, comps in pf:
        if comps == 3:
            out.append(f'        <DataArray type="Float64" Name="{name}" NumberOfComponents="3" format="ascii">\n')
            out += [f"          {f(v[0])} {f(v[1])} {f(v[2])}\n" for v in np.asarray(data, np.float64).reshape(-1, 3)]
            out.append("        </DataArray>\n")
    scalars = [(name, data) for name, data, comps in pf if comps == 1] + [(k, nodal[k]) for k in NODAL_NAMES]
    for name, data in scalars:
        out.append(f'        <DataArray type="Float64" Name="{name}" format="ascii">\n          ')
        out += [f(v) + " " for v in np.asarray(data, np.float64).reshape(-1)]
        out.append("\n        </DataArray>\n")
    out += ["      </PointData>\n", "    </Piece>\n", "  </UnstructuredGrid>\n", "</VTKFile>\n"]
    return "".join(out).encode()


def golden_module():
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden_vtu", os.path.join(HERE, "golden", "make_golden_vtu.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def golden_inputs(orc):
    import importlib.util
    spec = importlib.util.spec_from_file_location("make_golden_vtu", os.path.join(HERE, "golden", "make_golden_vtu.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    xyz, conn = orc.generate_cube(2, 1, 1, 1000.0, 800.0, 600.0)
    pf, cf = mod.fields(xyz, conn.shape[0])
    return xyz, conn, pf, cf


def attach(geo, mesh, pf, cf):
    for name, data, comps in pf:
        (mesh.field_data.add_field(geo.ScalarField(name, data)) if comps == 1
         else mesh.field_data.add_vector_field(geo.VectorField(name, data)))
    for name, data, comps in cf:
        (mesh.cell_data.add_field(geo.ScalarField(name, data)) if comps == 1
         else mesh.cell_data.add_vector_field(geo.VectorField(name, data)))


# ------------------------------------------------------------------------ CPU
def test_oracle_rust_display_known_answers(orc):
    f = orc.format_f64
    assert f(0.1 + 0.2) == "0.30000000000000004"
    assert f(1.0) == "1" and f(-1.5) == "-1.5" and f(100.0) == "100"
    assert f(0.0) == "0" and f(-0.0) == "-0"
    assert f(1e21) == "1" + "0" * 21 and f(1e-7) == "0.0000001"
    assert f(math.nan) == "NaN" and f(math.inf) == "inf" and f(-math.inf) == "-inf"
    assert f(5e-324) == "0." + "0" * 323 + "5"
    assert f(1.7976931348623157e308) == "17976931348623157" + "0" * 292
    assert f(2.2250738585072014e-308) == "0." + "0" * 307 + "22250738585072014"


def test_oracle_display_matches_repr(orc):
    for v in sample_doubles(20000):
        assert orc.format_f64(v) == rust_display_from_repr(float(v)), repr(v)


def test_oracle_writer_matches_python_restatement_and_golden(orc):
    xyz, conn, pf, cf = golden_inputs(orc)
    data = orc.write_vtu(xyz, conn, pf, cf)
    assert data == python_write_vtu(xyz, conn, pf, cf)
    with open(GOLDEN, "rb") as fh:
        assert fh.read() == data
    # no fields: no PointData / CellData blocks (vtk_writer.rs:175, :217)
    bare = orc.write_vtu(xyz, conn)
    assert b"PointData" not in bare and b"CellData" not in bare
    assert bare == python_write_vtu(xyz, conn, [], [])


def test_oracle_legacy_and_nodal_writers(orc):
    """VtkWriter::write and write_nodal_vtu: the oracle = a Python restatement = the golden files."""
    xyz, conn, pf, cf = golden_inputs(orc)
    plastic = golden_module().plastic_fields(conn.shape[0])
    legacy = orc.write_vtu(xyz, conn, pf, cf, fmt="legacy")
    assert legacy == python_write_vtk(xyz, conn, pf, cf)
    with open(os.path.join(HERE, "golden", "vtk_2x1x1.vtk"), "rb") as fh:
        assert fh.read() == legacy
    nodal = orc.write_vtu(xyz, conn, pf, cf + plastic, fmt="nodal")
    assert nodal == python_write_vtu_nodal(xyz, conn, pf, cf + plastic)
    with open(os.path.join(HERE, "golden", "vtu_nodal_2x1x1.vtu"), "rb") as fh:
        assert fh.read() == nodal
    # without PlasticStrain the reference leaves the other fields as sums (no count)
    assert orc.write_vtu(xyz, conn, pf, plastic[1:], fmt="nodal") == python_write_vtu_nodal(xyz, conn, pf,
                                                                                              plastic[1:])
    assert orc.write_vtu(xyz, conn, [], [], fmt="legacy") == python_write_vtk(xyz, conn, [], [])


def test_vtk_format_and_builder(geo):
    """vtk_writer.rs:1014-1075 (extension, format detection, recommended filename)."""
    F = geo.VtkFormat
    assert [F.extension(f) for f in (F.Legacy, F.Xml, F.XmlNodal, F.XmlMultiBlock)] == [".vtk", ".vtu", ".vtu", ".vtm"]
    assert F.from_filename("out/a.vtk") == F.Legacy and F.from_filename("a.vtu") == F.XmlNodal
    assert F.from_filename("a.vtm") == F.XmlMultiBlock and F.from_filename("a.txt") is None
    b = geo.VtkOutputBuilder(None)
    assert b.recommended_filename("out/step_0001") == "out/step_0001.vtu"
    assert b.with_format(F.Legacy).recommended_filename("x") == "x.vtk"
    b2 = geo.VtkOutputBuilder(None).with_tracers(object()).with_format(F.Legacy).with_fields(["T", "u"])
    assert b2.format == F.Legacy and b2.tracers is not None and len(b2.fields) == 2


def test_python_field_containers(geo):
    fd = geo.FieldData()
    assert fd.is_empty()
    fd.add_field(geo.ScalarField("T", np.zeros(4)))
    fd.add_vector_field(geo.VectorField.from_dof_vector("u", np.zeros(12)))
    assert fd.field_names() == ["T"] and fd.vector_field_names() == ["u"]
    assert fd.get_vector_field("u").len() == 4 and not fd.is_empty()
    with pytest.raises(geo.GeoError):
        geo.VectorField.from_dof_vector("bad", np.zeros(4))


# ------------------------------------------------------------------------ GPU
@pytest.mark.gpu
def test_device_vtu_matches_golden_and_oracle(orc, geo):
    xyz, conn, pf, cf = golden_inputs(orc)
    mesh = geo.Mesh(xyz, conn.astype(np.int32))
    attach(geo, mesh, pf, cf)
    data = geo.VtkWriter.render_vtu(mesh)
    with open(GOLDEN, "rb") as fh:
        assert data == fh.read()


@pytest.mark.gpu
def test_device_display_every_class_of_double(orc, geo):
    """A 1x1x1 mesh carrying long scalar and vector fields of sampled doubles (the
    writer prints a field's values whatever their count, vtk_writer.rs:186-188)."""
    xyz, conn = orc.generate_cube(1, 1, 1, 1.0, 1.0, 1.0)
    vals = sample_doubles(60000, seed=23)
    vecs = vals[: (vals.size // 3) * 3][::-1].copy()
    pf = [("bits", vals, 1), ("vec", vecs, 3)]
    mesh = geo.Mesh(xyz, conn.astype(np.int32))
    attach(geo, mesh, pf, [])
    assert geo.VtkWriter.render_vtu(mesh) == orc.write_vtu(xyz, conn, pf, [])


@pytest.mark.gpu
def test_device_vtu_sinks_agree_and_device_fields(orc, geo, tmp_path):
    import torch
    s = (6, 5, 4, 1000.0, 800.0, 600.0)
    dm = geo.ImprovedMeshGenerator.generate_cube_device(*s)
    xyz, conn = orc.generate_cube(*s)
    rng = np.random.default_rng(5)
    T = rng.normal(600.0, 300.0, xyz.shape[0])
    u = rng.normal(0.0, 1e-3, 3 * xyz.shape[0])
    dm.field_data.add_field(geo.ScalarField("T", torch.from_numpy(T).cuda()))
    dm.field_data.add_vector_field(geo.VectorField.from_dof_vector("u", torch.from_numpy(u).cuda()))
    host = geo.VtkWriter.render_vtu(dm)
    assert host == orc.write_vtu(xyz, conn, [("T", T, 1), ("u", u, 3)], [])
    dev = torch.empty(len(host), dtype=torch.uint8, device="cuda")
    assert geo.VtkWriter.render_vtu(dm, out=dev) == len(host)
    assert bytes(dev.cpu().numpy()) == host
    path = tmp_path / "out.vtu"
    assert geo.VtkWriter.write_vtu(dm, str(path)) == len(host)
    assert path.read_bytes() == host
    # the device mesh never came to the host
    assert dm._nodes is None and dm._elements is None
    small = np.empty(len(host) - 1, np.uint8)
    with pytest.raises(geo.GeoError):
        geo.VtkWriter.render_vtu(dm, out=small)


@pytest.mark.gpu
def test_device_vtu_streams_many_chunks_and_round_trips(geo, tmp_path):
    """64^3 cube (2.1M nodes, ~150 MB of text, several 64 MB chunks): the file equals
    the in-memory render, and every printed number reads back exactly."""
    n = 64
    dm = geo.ImprovedMeshGenerator.generate_cube_device(n, n, n, 1000.0, 1000.0, 600.0)
    rng = np.random.default_rng(9)
    T = rng.normal(600.0, 300.0, dm.num_nodes())
    dm.field_data.add_field(geo.ScalarField("Temperature", T))
    path = tmp_path / "big.vtu"
    size = geo.VtkWriter.write_vtu(dm, str(path))
    text = path.read_bytes()
    assert len(text) == size > (128 << 20)
    assert text == geo.VtkWriter.render_vtu(dm)
    parts = text.split(b"</DataArray>")
    pts = np.array(parts[0].split(b'format="ascii">\n', 1)[1].split(), np.float64).reshape(-1, 3)
    assert np.array_equal(pts.view(np.uint64), dm.nodes.view(np.uint64))
    ids = np.array(parts[1].split(b'format="ascii">\n', 1)[1].split(), np.int64)
    assert np.array_equal(ids, dm.elements.reshape(-1))
    temp = np.array(parts[4].split(b'format="ascii">\n', 1)[1].split(), np.float64)
    assert np.array_equal(temp.view(np.uint64), T.view(np.uint64))


@pytest.mark.gpu
def test_device_legacy_and_nodal_match_golden_and_oracle(orc, geo, tmp_path):
    xyz, conn, pf, cf = golden_inputs(orc)
    plastic = golden_module().plastic_fields(conn.shape[0])
    mesh = geo.Mesh(xyz, conn.astype(np.int32))
    attach(geo, mesh, pf, cf)
    with open(os.path.join(HERE, "golden", "vtk_2x1x1.vtk"), "rb") as fh:
        assert geo.VtkWriter.render_vtu(mesh, fmt=geo._native.GEO_VTK_LEGACY) == fh.read()
    attach(geo, mesh, [], plastic)
    nodal = geo.VtkWriter.render_vtu(mesh, fmt=geo._native.GEO_VTK_XML_NODAL)
    with open(os.path.join(HERE, "golden", "vtu_nodal_2x1x1.vtu"), "rb") as fh:
        assert nodal == fh.read()
    # the builder's default format and quick_write_vtu write the nodal file
    path = tmp_path / "step.vtu"
    assert geo.quick_write_vtu(mesh, str(path)) == len(nodal)
    assert path.read_bytes() == nodal
    legacy = tmp_path / "step.vtk"
    geo.VtkOutputBuilder(mesh).auto_format(str(legacy)).write(str(legacy))
    assert legacy.read_bytes() == orc.write_vtu(xyz, conn, pf, cf + plastic, fmt="legacy")
    with pytest.raises(geo.GeoError):
        geo.VtkOutputBuilder(mesh).with_format(geo.VtkFormat.XmlMultiBlock).write(str(tmp_path / "x.vtm"))


@pytest.mark.gpu
def test_device_nodal_averaging_larger_mesh(orc, geo):
    """8x6x5 device mesh, plasticity fields with and without PlasticStrain (sums vs
    averages), vector and scalar point fields from device memory."""
    import torch
    s = (8, 6, 5, 1000.0, 800.0, 600.0)
    dm = geo.ImprovedMeshGenerator.generate_cube_device(*s)
    xyz, conn = orc.generate_cube(*s)
    rng = np.random.default_rng(41)
    u = rng.normal(0.0, 1e-3, 3 * xyz.shape[0])
    T = rng.normal(600.0, 300.0, xyz.shape[0])
    plastic = golden_module().plastic_fields(conn.shape[0])
    for with_strain in (True, False):
        fields = plastic if with_strain else plastic[1:]
        dm.field_data = geo.FieldData()
        dm.cell_data = geo.FieldData()
        dm.field_data.add_vector_field(geo.VectorField.from_dof_vector("u", torch.from_numpy(u).cuda()))
        dm.field_data.add_field(geo.ScalarField("T", T))
        for name, data, _ in fields:
            dm.cell_data.add_field(geo.ScalarField(name, torch.from_numpy(data).cuda()))
        got = geo.VtkWriter.render_vtu(dm, fmt=geo._native.GEO_VTK_XML_NODAL)
        assert got == orc.write_vtu(xyz, conn, [("u", u, 3), ("T", T, 1)], fields, fmt="nodal")
        legacy = geo.VtkWriter.render_vtu(dm, fmt=geo._native.GEO_VTK_LEGACY)
        assert legacy == orc.write_vtu(xyz, conn, [("u", u, 3), ("T", T, 1)], fields, fmt="legacy")

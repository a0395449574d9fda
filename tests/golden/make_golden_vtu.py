"""Generates tests/golden/vtu_2x1x1.vtu, vtk_2x1x1.vtk and vtu_nodal_2x1x1.vtu:
VtkWriter::write_vtu (mesh/vtk_writer.rs:104-265), VtkWriter::write (:13-101) and
VtkWriter::write_nodal_vtu (:531-789) of the 2x1x1 ImprovedMeshGenerator cube with
two point fields and two cell fields (plus the plasticity cell fields for the nodal file),
from the CPU oracle (oracle/vtu.cpp), whose number formatting is checked against
Python's repr (an independent shortest round-trip implementation) in
tests/test_vtu.py. Regenerate with:
    python tests/golden/make_golden_vtu.py
"""
import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle import oracle as orc  # noqa: E402


def fields(xyz, n_elem):
    """Seeded fields with awkward decimals, negative values, a zero, -0.0 and a subnormal."""
    x, y, z = xyz[:, 0], xyz[:, 1], xyz[:, 2]
    temperature = 1280.0 * (1.0 - z / 600.0) + 1e-3 * x / 7.0
    disp = np.stack([1e-5 * np.sin(x / 100.0), -2.5e-6 * y / 3.0, -1e-4 * z / 600.0], 1)
    rng = np.random.default_rng(17)
    k = np.exp(rng.normal(np.log(3.0), 0.5, n_elem))
    k[0], k[1] = 0.0, -0.0
    flux = rng.normal(0.0, 1.0, (n_elem, 3)) * np.array([1e300, 1e-300, 1.0])
    flux[2, 0] = 5e-324
    return ([("Temperature", temperature, 1), ("Displacement", disp, 3)],
            [("Conductivity", k, 1), ("HeatFlux", flux, 3)])


NODAL_NAMES = ["PlasticStrain", "Stress_II", "StrainRate_II", "Pressure", "Viscosity", "IsYielding",
               "YieldStress", "PlasticViscosity", "SoftenedCohesion"]


def plastic_fields(n_elem, with_strain=True):
    """Seeded plasticity cell fields read by write_nodal_vtu (all but Viscosity present)."""
    rng = np.random.default_rng(29)
    out = [(name, rng.lognormal(0.0, 1.0, n_elem) * 10.0 ** (k - 4), 1)
           for k, name in enumerate(NODAL_NAMES) if name != "Viscosity"]
    return out if with_strain else out[1:]


def main():
    xyz, conn = orc.generate_cube(2, 1, 1, 1000.0, 800.0, 600.0)
    pf, cf = fields(xyz, conn.shape[0])
    outputs = {
        "vtu_2x1x1.vtu": orc.write_vtu(xyz, conn, pf, cf),
        "vtk_2x1x1.vtk": orc.write_vtu(xyz, conn, pf, cf, fmt="legacy"),
        "vtu_nodal_2x1x1.vtu": orc.write_vtu(xyz, conn, pf, cf + plastic_fields(conn.shape[0]), fmt="nodal"),
    }
    for name, data in outputs.items():
        with open(os.path.join(HERE, name), "wb") as fh:
            fh.write(data)
        print(name, len(data), "bytes")


if __name__ == "__main__":
    main()

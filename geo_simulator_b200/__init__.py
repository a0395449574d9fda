"""geo_simulator_b200 -- B200-native (sm_100a) Tet10 FEM hot path of GeoSimulator.

Element integration, deterministic CSR assembly with Dirichlet elimination,
Neumann flux boundary conditions on Tet10 faces,
Jacobi-PCG (FP64 drop-in), a matrix-free operator with a persistent PCG
(FP64 and mixed FP32/FP64), and a hand-written adjoint, all behind the C ABI
of ``include/geo_fem.h`` (``libgeofem.so``).
"""
from .fem import (  # noqa: F401
    Assembler, BodyForce, BoundaryConditions, BoundaryFace, ConjugateGradient, Context, CsrMatrix, DofManager,
    ElasticityElement, ElasticityOperator, ElementMatrix, GeoError, ImprovedMeshGenerator, IsotropicElasticity,
    MaxwellViscoelasticity, Mesh, DeviceMesh, NeumannBC, SolverStats, StressHistory, Tet10Face, ThermalOperator, BackwardEuler,
    TimeStepStats, update_stresses_maxwell, FieldData, ScalarField, VectorField, VtkWriter,
    VtkFormat, VtkOutputBuilder, quick_write_vtu, BiCGSTAB, GMRES, DirectSolver,
)

__version__ = "0.1.0"

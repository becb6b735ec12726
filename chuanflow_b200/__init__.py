"""chuanflow_b200: ChuanFlow's 3D unstructured finite-volume SIMPLE path on one
NVIDIA B200 (sm_100a).

The work happens in libchuanflow_b200.so (C++ host + CUDA kernels) behind the
C ABI declared in include/chuanflow_b200.h.  This module is a thin ctypes
view of that ABI, shaped after the reference's C++ interface:

    PolyMesh                      polyMesh / BlockMesh::create (src/3d/.../PolyMesh.h, BlockMesh.h)
    SimpleCase                    volVectorField U, volScalarField p, surfaceScalarField phi + Schemes
    SimpleCase.solve(controls)    solveIncompressibleSimple (src/3d/.../SimpleSolver.h:119-127)
    solve_cg / solve_bicgstab     solveCG / solveBiCGStab (src/common/.../Matrix.h:67-73)

There is no CPU fallback: importing the package without the built library,
or running it without a CUDA device, raises.
"""
from ._capi import (  # noqa: F401
    BC,
    DIV,
    Batch,
    GRAD,
    CfgError,
    PisoControls,
    PolyMesh,
    Schemes,
    SimpleCase,
    SimpleControls,
    SimpleResult,
    SolverReport,
    lib,
    inspect_case_file,
    lib_path,
    run_case_file,
    solve_bicgstab,
    solve_cg,
)

__all__ = ["BC", "Batch", "DIV", "GRAD", "CfgError", "PisoControls", "PolyMesh", "Schemes", "SimpleCase", "SimpleControls",
           "SimpleResult", "SolverReport", "inspect_case_file", "lib", "lib_path", "run_case_file", "solve_bicgstab", "solve_cg"]

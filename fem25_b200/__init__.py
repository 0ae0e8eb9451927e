"""fem25_b200 -- B200 (sm_100a) implementation of the fem25 hot path.

Python host side of ``libfem25gpu.so`` (the C ABI in ``include/fem25gpu.h``).
The entry points mirror the reference Fortran routines they replace:

    graph_build(mesh)                  GEN_GRAPH25        graph25_driver.f90:2
    Context.asmble_driver(...)         ASMBLE_DRIVER      asmble.f90:1
    Context.assemble(...)              ASMBLE_DRIVER into complex128 / complex64 device CSR
    Context.assemble_batch(...)        many (omega, py) systems per call (streaming launches of
                                       up to min(nslots, 1024) systems each)
    Context.asmb_peff(...)             ASMB_PEFF          asmble.f90:318
    Context.gradient(...)              exact adjoint gradient in lambda, mu, rho
    Context.cfmat_adjgrad(...)         CFMAT_DIST + ADJFLAM_DIST (reference-compatible)
    Context.misfit(...)                EXRESP25D + COBJ4 + BPRESID4 + RESID_DRHS
    Context.postsolve(...)             ADDBLK + the misfit pass, one kernel

Errors follow the reference's IERR convention: a nonzero status raises
``Fem25Error`` carrying the status code and the library's message.  There is
no CPU fallback: without the CUDA library every call fails.
"""
from .lib import (FEM25_PREC_FP64, FEM25_PREC_TF32X3, FEM25_PREC_TF32X3_POINTWISE, Context,
                  Fem25Error, graph_build, lib, fazmod, mesh_struct, read_mesh, sparse_plan)

__all__ = ["Context", "Fem25Error", "fazmod", "graph_build", "lib", "mesh_struct", "read_mesh",
           "sparse_plan", "FEM25_PREC_FP64", "FEM25_PREC_TF32X3", "FEM25_PREC_TF32X3_POINTWISE"]

"""mex_linear_algebra_b200 -- GF(2) linear algebra on B200 (sm_100a).

A drop-in for the six MEX functions of HCPhy/mex_linear_algebra
(``mela_matmul_gf2/_m4ri``, ``mela_rank_gf2/_m4ri``, ``mela_null_gf2/_m4ri``).
Every computation runs in the CUDA library ``libmela_b200.so`` through its C
ABI (include/mela.h); this module is the Python face of that ABI:

* ``mex_linear_algebra_b200.mela`` -- the six functions with MATLAB
  semantics on numpy arrays (column-major logical / double in, logical or
  double out, the reference's error messages);
* ``mex_linear_algebra_b200.device`` -- packed, stream-ordered device entry
  points over torch CUDA tensors (memory and streams only).
"""
from ._lib import lib, MelaError, check  # noqa: F401

__all__ = ["lib", "MelaError", "check"]

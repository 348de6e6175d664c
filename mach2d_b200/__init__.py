"""mach2d_b200 -- MACH-2D's SIMPLEC outer iteration on NVIDIA B200 (sm_100a).

The CUDA kernels and the C ABI live in libmach2d_b200.so (csrc/, declared in
include/mach2d_b200.h); this package is the host-side mirror of the
reference's interfaces:

  solvers        class_solver_msi5d/9d, class_solver_tdma5d/9d, solvers_init,
                 norm_l1_* (src/solvers/)
  coefficients   the routines of module coefficients and of the internal-flow
                 plug-in (src/equations/mach2d_coef.f90,
                 src/user/internal_flow/mod_intflow.f90)
  simplec        the device-resident outer iteration (src/mach2d_main.f90),
                 batches of instances
  ifile          reader for the reference's `value & name & description` decks
  thermo         the gas-mixture model (src/thermophysical/) and its data files
  listing        the reference's residual listing and main-results report
  sweep          sweeps of independent nozzles sharded over GPUs
  unet           the learned p' correction (no counterpart in the reference)
"""
from ._lib import LIB_PATH, M2DError, lib  # noqa: F401


def build(force=False):
    """Compiles libmach2d_b200.so in-tree (nvcc, sm_100a)."""
    from .build import build as _build
    return _build(force=force)

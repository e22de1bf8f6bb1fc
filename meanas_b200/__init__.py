"""B200-native FDFD solve path: a drop-in for ``meanas.fdfd.solvers.generic``.

Modules:

* ``solvers``    ``generic()`` with the reference's signature.
* ``operators``  ``GridOperator``: the device-resident wave operator and its solver.
* ``scpml``      SC-PML cell widths (``prepare_s_function``, ``stretch_with_scpml``, ...).
* ``fields``     sources before the solve and E -> H / Poynting after it.
* ``waveguide``  unidirectional waveguide-mode sources (``expand_e``, ``compute_source``).
* ``csr``        the GPU solver for the reference's ``matrix_solver`` hook.
* ``fdtd``       FDTD Yee updates with CPML.
* ``autograd``   ``fdfd_solve``: dL/d(epsilon) through the adjoint solve.
* ``serving``    continuous-batching request server.
* ``workloads``  seeded synthetic problems of the benchmark shapes.
* ``build``      the nvcc recipe for ``libmeanas_fdfd.so`` (sm_100a).
"""
from . import scpml  # noqa: F401

__all__ = ['generic', 'GridOperator', 'last_solve_info', 'scpml']


def __getattr__(name):
    if name in ('generic', 'last_solve_info'):
        from . import solvers
        return getattr(solvers, name)
    if name == 'GridOperator':
        from .operators import GridOperator
        return GridOperator
    raise AttributeError(name)

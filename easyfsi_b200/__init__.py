"""easyfsi_b200: B200-native (sm_100a) implementation of the EasyFsi coupled-step
hot path -- graded-grid pressure projection, neo-Hookean MPM substep and HIBM
force spreading -- behind the reference's Python entry points.

Modules mirror the reference's layout: ``fluid`` (CartesianFluidSolver and the
grid classes), ``neo_hookean_mpm`` (NeoHookeanMpmState), ``hibm_mpm``
(HibmMpmSurfaceMarkers), ``hyperelastic``, ``geometry`` and ``runtime``.  The
numerical work runs in ``libeasyfsi_b200.so`` (C ABI in include/easyfsi_b200.h).
"""

__version__ = "0.1.0"

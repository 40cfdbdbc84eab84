"""pywrf_b200: B200-native (sm_100a) ARW integration step with PyWRF's call surface.

``WrfSolver`` is the drop-in for ``pywrf.WrfSolver`` (construct, then
``solve()``); ``wrf_physics.wsm6`` and ``wrf_dynamics.advect_scalar`` take the
reference functions' arguments.  The kernels live in the in-tree library
``pywrf_b200/lib/libpywrf_b200.so`` (``python -m pywrf_b200.build``).
"""
__version__ = "0.1.0"


def __getattr__(name):
    if name in ("WrfSolver", "Integrator"):
        from . import solver
        return getattr(solver, name)
    raise AttributeError(name)


__all__ = ["WrfSolver", "Integrator"]

"""B200-native (sm_100a, FP64) time-stepping path of StaRMAP.

Public API mirrors the reference: ``par = starmap_init(prob)`` and
``output = starmap_solver(par)``; the time loop runs in ``libstarmap_gpu.so``.
"""
from .closure import closure, closure_pn, closure_spn
from .init import capargs, hook, nargin, starmap_init, zero

__all__ = ["closure", "closure_pn", "closure_spn", "starmap_init", "nargin", "capargs", "zero", "hook",
           "starmap_solver"]


def starmap_solver(par):
    from .solver import starmap_solver as _run
    return _run(par)

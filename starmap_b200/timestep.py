"""Parabolic time-step selection of ``starmap_solver.m`` (``par.timestep`` 1 or 2).

With ``timestep > 0`` the reference does not use the hyperbolic step
``dt_hyp``; it searches the largest dt for which the von Neumann growth
matrix of one full step, built from the smallest absorption and total
cross-sections, has spectral radius below ``la0 = 1 + 1e-8``
(starmap_solver.m:173-203): starting from ``max(dt, dt_hyp)`` it doubles or
halves until the bracket straddles ``la0`` (lowering ``la0`` to 1 once a
strictly contracting step is seen), then bisects geometrically until the
bracket's ratio reaches 0.98, unless the bracket's lower end already exceeds
the time left.  For time-dependent materials the search runs every step and
the averaged materials fall back to those at time t when they are unstable
with the chosen dt (:253-265).  Autonomous problems search once, at the
first step.

The search itself runs on the host; each trial's growth matrix is formed
on the host (n_sys^2 work) and its spectral radius -- three n_sys^3 complex
products and the dense complex eigenvalues of the reference's ``eig`` -- is
computed on the GPU (``smg_growth_radius``: cuBLAS and cuSOLVER) when a
CUDA device is present, else with numpy.  The device only receives the
resulting dt.
"""
from __future__ import annotations

import numpy as np

__all__ = ["symbol", "decay_vector", "growth_factor", "search", "stable", "use_device_eigenvalues"]

LA0 = 1 + 1e-8
_DEVICE = None   # None: decided at the first growth factor (a CUDA device is present)


def use_device_eigenvalues(flag=None):
    """Compute growth-matrix spectral radii on the GPU (True), with numpy
    (False), or on the GPU when a CUDA device is present (None, default)."""
    global _DEVICE
    _DEVICE = flag


def _device_enabled() -> bool:
    global _DEVICE
    if _DEVICE is None:
        try:
            from . import _lib
            _DEVICE = _lib.lib().smg_device_count() > 0
        except Exception:
            _DEVICE = False
    return bool(_DEVICE)


def _device_radius(G, odd) -> float:
    import ctypes as C

    from . import _lib
    n = G.shape[0]
    Gc = np.asfortranarray(G, dtype=np.complex128)
    mask = np.zeros(n, dtype=np.int32)
    mask[list(odd)] = 1
    la = C.c_double()
    _lib.check(_lib.lib().smg_growth_radius(n, Gc.ctypes.data_as(C.POINTER(C.c_double)),
                                            mask.ctypes.data_as(C.POINTER(C.c_int32)), C.byref(la)))
    return float(la.value)


def symbol(Mx, My, Mz, h):
    """``M = -1i*(Mx/h(1) + My/h(2) + Mz/h(3))`` (starmap_solver.m:108)."""
    return -1j * (np.asarray(Mx) / h[0] + np.asarray(My) / h[1] + np.asarray(Mz) / h[2])


def _first_nonsingleton_min(A):
    A = np.asarray(A, dtype=np.float64)
    for d, n in enumerate(A.shape):
        if n != 1:
            return np.min(A, axis=d, keepdims=True)
    return A


def _min_min(A) -> float:
    """MATLAB ``min(min(A))`` for a coefficient array: a scalar for 1D/2D
    fields; a 3D field with several planes leaves a vector, which the
    reference cannot store in ``decay(j)`` (it stops with an error)."""
    v = _first_nonsingleton_min(_first_nonsingleton_min(A))
    if v.size != 1:
        raise ValueError("parabolic time step: min(min(.)) of a 3D coefficient field is not a scalar "
                         "(starmap_solver.m:175-179 fails for such fields)")
    return float(v.reshape(()))


def decay_vector(n_sys, gt, mom_order, sA111, sT):
    """Smallest sigma_a for component 1 and smallest sigma_t of each other
    component's (grid type, order) (starmap_solver.m:175-179)."""
    decay = np.ones(n_sys) * _min_min(sA111)
    for j in range(1, n_sys):
        decay[j] = _min_min(sT[(int(gt[j, 0]), int(gt[j, 1]), int(gt[j, 2]), int(mom_order[j]))])
    return decay


def growth_factor(M, even, odd, decay, dt, timestep) -> float:
    """Spectral radius of the full-step growth matrix (starmap_solver.m:506-514).

    ``even``/``odd`` are the component indices updated by phase B and phase A;
    each half-update leaves the other set's rows at the identity, and one
    step is ``G_o G_e G_e G_o``.  ``timestep == 2`` measures growth relative
    to the decay ``exp(-decay(1) dt)``."""
    decay = np.asarray(decay, dtype=np.float64)
    # expm1div with the reference's Taylor branch (starmap_solver.m:531-535)
    x = -decay * dt / 2
    phi = 1 + x * .5 + x ** 2 / 6
    big = np.abs(x) > 2e-4
    phi[big] = (np.exp(x[big]) - 1) / x[big]
    G = (dt * phi)[:, None] * (M + np.diag(-decay / 2))
    n = len(decay)
    if _device_enabled():
        la = _device_radius(G, odd)
        if timestep == 2:
            la *= float(np.exp(decay[0] * dt))
        return la
    diag = (np.arange(n), np.arange(n))
    Ge = G.copy()
    Ge[odd, :] = 0
    Ge[diag] += 1
    Go = G.copy()
    Go[even, :] = 0
    Go[diag] += 1
    la = float(np.max(np.abs(np.linalg.eigvals(Go @ Ge @ Ge @ Go))))
    if timestep == 2:
        la *= float(np.exp(decay[0] * dt))
    return la


def search(M, even, odd, decay, dt_prev, dt_hyp, tleft, timestep):
    """Lower end of the final dt bracket and the threshold used
    (starmap_solver.m:174-203).  The caller takes ``min(dt, tleft)*cn``."""
    gf = lambda d: growth_factor(M, even, odd, decay, d, timestep)
    dt = max(dt_prev, dt_hyp)
    la = gf(dt)
    dt_br = [dt, dt]
    la_br = [la, la]
    la0 = LA0
    while ((la_br[0] < la0) == (la_br[1] < la0)) and (dt_br[0] <= tleft or la_br[0] > la0):
        ind = int(la_br[0] < la0) + 1            # 1: dt(1) unstable, 2: stable
        base = dt_br[ind - 1]
        dt_br = [base * 2.0 ** (ind - 2), base * 2 * 2.0 ** (ind - 2)]
        la_br = [la_br[1], la_br[0]]
        la_br[ind - 1] = gf(dt_br[ind - 1])
        if min(la_br) < 1:
            la0 = 1.0
    while dt_br[0] / dt_br[1] < 0.98 and dt_br[0] <= tleft:
        dt_mid = float(np.sqrt(dt_br[0] * dt_br[1]))
        la_mid = gf(dt_mid)
        ind = 1 + int(la_mid >= la0)
        dt_br[ind - 1] = dt_mid
        la_br[ind - 1] = la_mid
    return dt_br[0], la0


def stable(M, even, odd, decay, dt, la0, timestep) -> bool:
    """Whether the averaged materials are stable with dt (starmap_solver.m:260-262)."""
    return growth_factor(M, even, odd, decay, dt, timestep) < la0

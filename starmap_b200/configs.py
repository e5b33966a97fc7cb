"""Synthetic problem definitions (``prob`` dicts) for the benchmark workloads.

No public dataset exists for StaRMAP; these follow the shapes of the
reference's own example scripts with seeded, deterministic inputs:

* :func:`linesource` -- 2D P_N Gaussian line source (starmap_2d_ex_linesource.m:41-73
  template; periodic, sigma_a=0, sigma_s0=1).
* :func:`lattice` -- 2D checkerboard lattice (starmap_2d_ex_lattice.m:29-64) with the
  exponential moment filter of starmap_2d_ex_lattice_filter_convergence.m:143-147.
* :func:`pointsource3d` -- 3D P_N point source (starmap_3d_ex_pointsource.m:42-75
  template) with anisotropic scattering sigma_sm = 0.5^m and the filter.

The time step is realised through the reference's own knob: ``cn`` is chosen
so that ``dt = cn * dt_hyp`` equals ``0.5 * h``.  Discontinuous material data
is defined by which unit square a point lies in with a 1e-9 guard at the
square edges, so that staggered points lying exactly on an edge are assigned
as exact arithmetic would assign them.
"""
from __future__ import annotations

import numpy as np

from .closure import closure

EPS = np.finfo(float).eps


def _dt_hyp(closure_name, n_mom, dim, h):
    _, _, _, Mz = closure(closure_name, n_mom, dim)
    lam = np.max(np.abs(np.linalg.eigvals(Mz)))
    return min(h) / lam / {1: 1, 2: 2, 3: 3}[dim]


def cn_for_dt(closure_name, n_mom, dim, h, dt):
    return dt / _dt_hyp(closure_name, n_mom, dim, h)


def exp_filter(order: int, f_eff: float):
    """Reference exponential filter (starmap_2d_ex_lattice_filter_convergence.m:143-147)."""
    def f(par, dt, k):
        p = order
        N = par["n_mom"]
        f_b = -f_eff / np.log(np.exp(np.log(EPS) * (N / (N + 1)) ** p))
        return np.exp(np.log(EPS) * (k / (N + 1)) ** p) ** (dt * f_b)
    return f


def linesource(n=100, n_mom=7, tfinal=1.0, closure_name="P", std=0.03, bc=0):
    """2D P_N line source: Gaussian IC with std `std`, periodic, sigma_a=0, sigma_s0=1."""
    ax = [-1.5, 1.5, -1.5, 1.5]
    h = (ax[1] - ax[0]) / n
    return dict(
        name="Line Source", closure=closure_name, n_mom=n_mom, ax=ax, n=[n, n], bc=[bc, bc],
        ic=lambda x, y: np.exp(-(x ** 2 + y ** 2) / (2 * std ** 2)) / (2 * np.pi * std ** 2),
        sigma_a=lambda x, y: 0.0, sigma_s0=lambda x, y: 1.0,
        t_plot=[0.0, tfinal], tfinal=tfinal, cn=cn_for_dt(closure_name, n_mom, 2, [h, h], 0.5 * h),
        quiet=True)


def _lattice_mask(x, y):
    cx = np.ceil(x - 1e-9)
    cy = np.ceil(y - 1e-9)
    s = cx + cy
    return (np.ceil(s / 2) * 2 == s) & (1 < cx) & (cx < 7) & (1 < cy) & (cy - 2 * np.abs(cx - 4) < 4)


def lattice(n=350, n_mom=39, tfinal=3.2, filter_order=4, f_eff=10.0, f_position="substep", closure_name="P"):
    """2D checkerboard lattice with source q=1 in the central square, exp filter."""
    ax = [0.0, 7.0, 0.0, 7.0]
    h = 7.0 / n

    def sigma_a(x, y):
        g = _lattice_mask(x, y)
        return (1 - g) * 0 + g * 10.0

    def sigma_s0(x, y):
        g = _lattice_mask(x, y)
        return (1 - g) * 1.0 + g * 0

    def source(x, y):
        return ((3 + 1e-9 < x) & (x < 4 - 1e-9) & (3 + 1e-9 < y) & (y < 4 - 1e-9)).astype(np.float64)

    prob = dict(
        name="Lattice Test", closure=closure_name, n_mom=n_mom, sigma_a=sigma_a, sigma_s0=sigma_s0,
        source=source, ax=ax, n=[n, n], bc=[1, 1], t_plot=[0.0, tfinal], tfinal=tfinal,
        cn=cn_for_dt(closure_name, n_mom, 2, [h, h], 0.5 * h), quiet=True)
    if f_position:
        prob.update(filterfunction=exp_filter(filter_order, f_eff), f_position=f_position)
    return prob


def pointsource3d(n=128, n_mom=9, tfinal=0.75, std=0.05, filter_order=4, f_eff=10.0, f_position="substep"):
    """3D P_N point source, periodic, sigma_a=0.01, sigma_s0=1, sigma_sm=0.5^m, filter."""
    ax = [-1.0, 1.0, -1.0, 1.0, -1.0, 1.0]
    h = 2.0 / n
    prob = dict(
        name="Point Source", closure="P", n_mom=n_mom, ax=ax, n=[n, n, n], bc=[0, 0, 0],
        ic=lambda x, y, z: np.exp(-(x ** 2 + y ** 2 + z ** 2) / (2 * std ** 2)) / (2 * np.pi * std ** 2) ** 1.5,
        sigma_a=lambda x, y, z: 0.01, sigma_s0=lambda x, y, z: 1.0,
        sigma_sm=lambda x, y, z, m: 0.5 ** m,
        t_plot=[0.0, tfinal], tfinal=tfinal, cn=cn_for_dt("P", n_mom, 3, [h, h, h], 0.5 * h), quiet=True)
    if f_position:
        prob.update(filterfunction=exp_filter(filter_order, f_eff), f_position=f_position)
    return prob


def batched_sweep(n_inst=256, seed=20261203, edges=tuple(range(64, 257, 32)), orders=(3, 5, 7, 11, 15)):
    """Seeded batch of 2D P_N problems of uneven size and order.

    Grid edge uniform over ``edges``, N uniform over ``orders``; sigma_a and
    sigma_s0 piecewise constant on 8x8 blocks of [-1.5,1.5]^2 drawn
    log-uniformly in [0.01, 10]; Gaussian initial condition with a random
    centre in the inner 60% of the domain and standard deviation in
    [0.02, 0.1]; periodic; the reference's default CFL number (cn = 0.99).
    Returns a list of ``prob`` dicts (tfinal large: the batch is stepped a
    fixed number of steps)."""
    rng = np.random.default_rng(seed)
    probs = []
    for _ in range(n_inst):
        edge = int(rng.choice(edges))
        N = int(rng.choice(orders))
        sa = 10 ** rng.uniform(-2, 1, size=(8, 8))
        ss = 10 ** rng.uniform(-2, 1, size=(8, 8))
        cx, cy = rng.uniform(-0.9, 0.9, size=2)
        std = rng.uniform(0.02, 0.1)

        def block_field(tab):
            def f(x, y):
                i = np.clip(np.floor((x + 1.5) / 3.0 * 8).astype(int), 0, 7)
                j = np.clip(np.floor((y + 1.5) / 3.0 * 8).astype(int), 0, 7)
                return tab[i, j]
            return f

        def gaussian(cx, cy, std):
            return lambda x, y: np.exp(-((x - cx) ** 2 + (y - cy) ** 2) / (2 * std ** 2)) / (2 * np.pi * std ** 2)

        probs.append(dict(name="batch", closure="P", n_mom=N, ax=[-1.5, 1.5, -1.5, 1.5], n=[edge, edge],
                          bc=[0, 0], ic=gaussian(cx, cy, std), sigma_a=block_field(sa), sigma_s0=block_field(ss),
                          t_plot=[0.0, 1e9], tfinal=1e9, quiet=True))
    return probs


def adjoint_problem(n=200, n_mom=15, sigma_a_field=None):
    """2D P15 inverse-problem setting: [-1.5,1.5]^2, periodic, sigma_s0 = 1,
    normalised Gaussian initial condition with std 0.05, dt = 0.5 h.
    ``sigma_a_field(x, y)`` defaults to the constant 0.1 returned as an array
    (so that its gradient is a field); :func:`true_sigma_a` is the field that
    generates the observations."""
    ax = [-1.5, 1.5, -1.5, 1.5]
    h = 3.0 / n
    sa = sigma_a_field or (lambda x, y: 0.1 + 0.0 * x)
    std = 0.05
    return dict(name="Adjoint", closure="P", n_mom=n_mom, ax=ax, n=[n, n], bc=[0, 0],
                ic=lambda x, y: np.exp(-(x ** 2 + y ** 2) / (2 * std ** 2)) / (2 * np.pi * std ** 2),
                sigma_a=sa, sigma_s0=lambda x, y: 1.0, t_plot=[0.0, 1e9], tfinal=1e9,
                cn=cn_for_dt("P", n_mom, 2, [h, h], 0.5 * h), quiet=True)


def true_sigma_a(x, y):
    """0.1 plus two Gaussian bumps of amplitude 1 and std 0.2 at (+-0.5, 0)."""
    return 0.1 + np.exp(-((x - 0.5) ** 2 + y ** 2) / (2 * 0.2 ** 2)) + \
        np.exp(-((x + 0.5) ** 2 + y ** 2) / (2 * 0.2 ** 2))

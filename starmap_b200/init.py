"""``par = starmap_init(prob)``: problem normalisation in front of the solver.

Mirrors ``starmap_init.m`` of StaRMAP v2.0 for a Python host: ``prob`` and
``par`` are dicts whose keys are the reference's struct fields, hooks are
Python callables with the reference's argument conventions (README.txt:100-159)
and MATLAB's ``nargin`` is recovered from the callable's signature
(:func:`nargin`).  1D and 2D hooks are wrapped into the solver's 3D signature
exactly as starmap_init.m:75-208 does, so that the solver always sees
``(x, y, z, ...)`` with the first axis a singleton in 2D.
"""
from __future__ import annotations

import inspect

import numpy as np

from .closure import closure

__all__ = ["starmap_init", "nargin", "capargs", "zero", "hook"]


def nargin(fct) -> int:
    """MATLAB ``nargin(fct)``: declared argument count, negative for varargs.

    A callable may carry an explicit ``_nargin`` attribute (set by
    :func:`hook`); otherwise positional parameters are counted and a
    ``*args`` parameter gives ``-(count + 1)`` like MATLAB's ``varargin``.
    """
    n = getattr(fct, "_nargin", None)
    if n is not None:
        return int(n)
    sig = inspect.signature(fct)
    count = 0
    for p in sig.parameters.values():
        if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD):
            count += 1
        elif p.kind == p.VAR_POSITIONAL:
            return -(count + 1)
    return count


def hook(fct, n: int):
    """Wrap ``fct`` so that :func:`nargin` reports ``n``."""
    def wrapped(*args):
        return fct(*args)
    wrapped._nargin = int(n)
    wrapped.__wrapped_hook__ = fct
    return wrapped


def capargs(fct, *args):
    """Call ``fct`` with as many arguments as it takes (starmap_solver.m:521-525)."""
    narg = max(nargin(fct), 1)
    return fct(*args[:narg])


def zero(*args):
    """Zero function (starmap_init.m:236-238): zeros shaped like the first argument."""
    return np.zeros(np.shape(args[0]))


def _noop_output(*args):
    return None


def _wrap(name, f, table):
    """Re-sign a user hook by its arity; ``table`` maps user nargin -> (solver nargin, adaptor)."""
    n = nargin(f)
    if n not in table:
        raise ValueError(f"{name} has incompatible number of arguments.")
    solver_n, adapt = table[n]
    return hook(adapt(f), solver_n)


def starmap_init(prob: dict) -> dict:
    """Configure ``par`` for :func:`starmap_b200.starmap_solver` (starmap_init.m:30-231)."""
    par = dict(prob)
    par["prob"] = dict(prob)
    # dimension detection and compatibility (starmap_init.m:36-60)
    if "ax" in prob:
        par["dim"] = len(prob["ax"]) // 2
    elif "n" in prob:
        par["dim"] = len(prob["n"])
    elif "bc" in prob:
        par["dim"] = len(prob["bc"])
    else:
        raise ValueError("At least one of ax, n, or bc should be defined")
    if "ax" in prob:
        if "n" in prob and len(prob["ax"]) / 2 != len(prob["n"]):
            raise ValueError("Incompatible problem variables ax and n.")
        if "bc" in prob and len(prob["ax"]) / 2 != len(prob["bc"]):
            raise ValueError("Incompatible problem variables ax and bc.")
    elif "n" in prob and "bc" in prob and len(prob["n"]) != len(prob["bc"]):
        raise ValueError("Incompatible problem variables n and bc.")

    # moment matrices (starmap_init.m:64-70)
    mo, Mx, My, Mz = closure(par["closure"], par["n_mom"], par["dim"])
    par["mom_order"], par["Mx"], par["My"], par["Mz"] = mo, Mx, My, Mz
    n_sys = Mz.shape[0]

    dim = par["dim"]
    if dim == 1:
        if "ax" in prob:
            par["ax"] = list(prob["ax"]) * 3
        if "n" in prob:
            par["n"] = [1, 1, int(np.atleast_1d(prob["n"])[0])]
        if "bc" in prob:
            b = int(np.atleast_1d(prob["bc"])[0])
            par["bc"] = [b, b, b]
        if "ic" in prob:
            par["ic"] = _wrap("ic", prob["ic"], {
                1: (3, lambda f: lambda _a, _b, x: f(x)),
                2: (4, lambda f: lambda _a, _b, x, k: f(x, k))})
        for key in ("sigma_a", "sigma_s0"):
            if key in prob:
                par[key] = _wrap(key, prob[key], {
                    1: (3, lambda f: lambda _a, _b, x: f(x)),
                    2: (4, lambda f: lambda _a, _b, x, t: f(x, t))})
        if "sigma_sm" in prob:
            # starmap_init.m:108-109 keeps the reference's (~,~,m,x) -> (x,m) mapping
            par["sigma_sm"] = _wrap("sigma_sm", prob["sigma_sm"], {
                2: (4, lambda f: lambda _a, _b, m, x: f(x, m)),
                3: (5, lambda f: lambda _a, _b, x, m, t: f(x, m, t))})
        if "source" in prob:
            par["source"] = _wrap("source", prob["source"], {
                2: (4, lambda f: lambda _a, _b, x, t: f(x, t)),
                3: (5, lambda f: lambda _a, _b, x, t, k: f(x, t, k)),
                1: (3, lambda f: lambda _a, _b, x: f(x))})
        if "filterfunction" in prob:
            par["filterfunction"] = _wrap("filterfunction", prob["filterfunction"], {
                4: (6, lambda f: lambda p, dt, k, _a, _b, x: f(p, dt, k, x)),
                5: (7, lambda f: lambda p, dt, k, _a, _b, x, t: f(p, dt, k, x, t)),
                3: (3, lambda f: f)})
        par.setdefault("output", _noop_output)
    elif dim == 2:
        if "ax" in prob:
            ax = list(prob["ax"])
            par["ax"] = ax[0:2] + ax
        if "n" in prob:
            par["n"] = [1] + [int(v) for v in prob["n"]]
        if "bc" in prob:
            b = [int(v) for v in prob["bc"]]
            par["bc"] = [b[0]] + b
        if "ic" in prob:
            par["ic"] = _wrap("ic", prob["ic"], {
                2: (3, lambda f: lambda _a, x, y: f(x, y)),
                3: (4, lambda f: lambda _a, x, y, k: f(x, y, k))})
        for key in ("sigma_a", "sigma_s0"):
            if key in prob:
                par[key] = _wrap(key, prob[key], {
                    2: (3, lambda f: lambda _a, x, y: f(x, y)),
                    3: (4, lambda f: lambda _a, x, y, t: f(x, y, t))})
        if "sigma_sm" in prob:
            par["sigma_sm"] = _wrap("sigma_sm", prob["sigma_sm"], {
                3: (4, lambda f: lambda _a, x, y, m: f(x, y, m)),
                4: (5, lambda f: lambda _a, x, y, m, t: f(x, y, m, t))})
        if "source" in prob:
            par["source"] = _wrap("source", prob["source"], {
                3: (4, lambda f: lambda _a, x, y, t: f(x, y, t)),
                4: (5, lambda f: lambda _a, x, y, t, k: f(x, y, t, k)),
                2: (3, lambda f: lambda _a, x, y: f(x, y))})
        if "filterfunction" in prob:
            par["filterfunction"] = _wrap("filterfunction", prob["filterfunction"], {
                5: (6, lambda f: lambda p, dt, k, _a, x, y: f(p, dt, k, x, y)),
                6: (7, lambda f: lambda p, dt, k, _a, x, y, t: f(p, dt, k, x, y, t)),
                3: (3, lambda f: f)})
        par.setdefault("output", _noop_output)
    elif dim == 3:
        par.setdefault("output", _noop_output)
    else:
        raise ValueError("dimension must be 1, 2 or 3")

    # defaults (starmap_init.m:213-231)
    par.setdefault("name", "Output")
    par.setdefault("ic", zero)
    par.setdefault("sigma_a", zero)
    par.setdefault("sigma_s0", zero)
    par.setdefault("source", zero)
    if "source_ind" not in par:
        ns = nargin(par["source"])
        last = int(ns >= 0) + int(ns > 4) * (n_sys - 1)
        par["source_ind"] = np.arange(1, last + 1)
    par.setdefault("ax", [0, 1, 0, 1, 0, 1])
    par.setdefault("n", [100, 100, 100])
    par.setdefault("timestep", 0)
    par.setdefault("cn", 0.99)
    par.setdefault("bc", [0, 0, 0])
    par.setdefault("t_plot", np.arange(0, 11) / 10.0)
    if "tfinal" not in par:
        par["tfinal"] = float(np.atleast_1d(par["t_plot"])[-1])
    par.setdefault("mom_output", 1)
    par["closure_mod"] = "F" if "filterfunction" in par else ""
    return par

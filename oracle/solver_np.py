"""ORACLE (test infrastructure only) -- numpy restatement of starmap_solver.m.

This module is the CPU checker for the GPU time-stepping path.  Only the test
suite, ``__graft_entry__.smoke()`` and the CPU-baseline leg of ``bench.py`` may
import it; the product path (``starmap_b200``) never does.

It restates StaRMAP v2.0 ``starmap_solver.m`` statement by statement with
Octave's array semantics: 3D column-major component arrays of shape
``(s1, s2, s3)``, ``diff`` over the boundary-extension index vectors, the
``sumcell`` summation order, the ``expm1div`` branch at ``|x| > 2e-4`` and every
quirk of the loop (constant dt with overshoot for autonomous problems, the
filter substep index reused between phases, absorption-only zeroth moment).
Each block cites the reference lines it follows.

Parity status: the reference is MATLAB/GNU Octave only, no Octave or MATLAB
is installed where this code is developed and tested, and the reference ships no
stored outputs or golden vectors.  The restatement is therefore *parity
unpinned* with respect to Octave itself; it is pinned instead by the
reference's own known-answer properties (P_N == SP_N for isotropic data,
starmap_2d_ex_boxes.m:7-16), by an independent discrete-symbol (von Neumann)
check of the staggered update, and by agreement with the independent C
restatement in ``oracle/loop_ref.c``.

Scope: hyperbolic and parabolic dt (``par.timestep`` 0, 1, 2); autonomous and time-dependent
material hooks; filters ``''``, ``'substep'`` and ``'full'``; 1D/2D/3D; both
boundary conditions.  Plot callbacks are replaced by optional snapshot capture.
"""
from __future__ import annotations

import math
from dataclasses import dataclass, field

import numpy as np

EPS = np.finfo(float).eps


# --------------------------------------------------------------------------
# MATLAB helpers
# --------------------------------------------------------------------------
def nargin(fct) -> int:
    n = getattr(fct, "_nargin", None)
    if n is not None:
        return int(n)
    import inspect
    cnt = 0
    for p in inspect.signature(fct).parameters.values():
        if p.kind in (p.POSITIONAL_ONLY, p.POSITIONAL_OR_KEYWORD):
            cnt += 1
        elif p.kind == p.VAR_POSITIONAL:
            return -(cnt + 1)
    return cnt


def capargs(fct, *args):
    """starmap_solver.m:521-525."""
    return fct(*args[:max(nargin(fct), 1)])


def expm1div(x):
    """(exp(x)-1)/x with the reference's Taylor branch (starmap_solver.m:531-535)."""
    x = np.asarray(x, dtype=np.float64)
    y = 1 + x * .5 + x ** 2 / 6
    ind = np.abs(x) > 2e-4
    if y.ndim == 0:
        return np.float64((np.exp(x) - 1) / x) if ind else np.float64(y)
    y = y.copy()
    y[ind] = (np.exp(x[ind]) - 1) / x[ind]
    return y


def colon(a, d, b):
    """Octave range ``a:d:b`` (base + k*inc, last element clamped to the limit)."""
    n = int(math.floor((b - a) / d + 1e-10)) + 1
    if n <= 0:
        return np.zeros(0)
    v = a + np.arange(n) * d
    if n > 1:
        v[-1] = min(a + (n - 1) * d, b)
    return v


def _ones_like_nargin(*args):
    return 1.0


_ones_like_nargin._nargin = -1


def _zero(*args):
    return np.zeros(np.shape(args[0]))


_zero._nargin = -1


# --------------------------------------------------------------------------
# Solver restatement
# --------------------------------------------------------------------------
@dataclass
class OracleResult:
    output: list
    U: list
    step_count: int
    t: float
    dt: float
    snapshots: list = field(default_factory=list)
    setup: dict = field(default_factory=dict)
    dts: list = field(default_factory=list)       # dt of every step


def _mat_min(A):
    """MATLAB ``min(A)``: along the first non-singleton dimension."""
    A = np.asarray(A, dtype=np.float64)
    for d, n in enumerate(A.shape):
        if n != 1:
            return np.min(A, axis=d, keepdims=True)
    return A


def _min2(A):
    """``min(min(A))`` as the decay vector needs it (starmap_solver.m:175-179):
    a scalar for 2D arrays; a 3D array with several planes leaves a vector,
    which the reference cannot store into ``decay(j)``."""
    v = _mat_min(_mat_min(A))
    if v.size != 1:
        raise ValueError("min(min(.)) of a 3D coefficient field is not a scalar (the reference fails here too)")
    return float(v.reshape(()))


def _decay(sA, sT, n_sys, gtx, gty, gtz, mom_order):
    """Smallest absorption and total cross-sections per component
    (starmap_solver.m:175-179 and 255-259)."""
    decay = np.ones(n_sys) * _min2(sA)
    for j in range(1, n_sys):
        decay[j] = _min2(sT[int(gtx[j]), int(gty[j]), int(gtz[j]), int(mom_order[j])])
    return decay


def _growth_factor(Msym, c, decay, dt, timestep):
    """Largest eigenvalue modulus of the von Neumann growth matrix of one full
    step (starmap_solver.m:506-514): G = diag(dt*phi(-decay*dt/2))*(M -
    diag(decay/2)); the even update leaves the odd rows at the identity and
    vice versa; one step is G_o*G_e*G_e*G_o; timestep 2 scales by
    exp(decay(1)*dt)."""
    decay = np.asarray(decay, dtype=np.float64)
    G = np.diag(dt * expm1div(-decay * dt / 2)) @ (Msym + np.diag(-decay / 2))
    I = np.eye(len(decay))
    even = c["111"] + c["221"] + c["212"] + c["122"]
    odd = c["211"] + c["121"] + c["112"] + c["222"]
    Ge = G.copy()
    Ge[odd, :] = 0
    Ge = Ge + I
    Go = G.copy()
    Go[even, :] = 0
    Go = Go + I
    G = Go @ Ge @ Ge @ Go
    la = float(np.max(np.abs(np.linalg.eigvals(G))))
    if timestep == 2:
        la = la * np.exp(decay[0] * dt)
    return la


def _classify(Mx, My, Mz):
    """Grid-type classification (starmap_solver.m:76-98)."""
    n_sys = Mz.shape[0]
    Ix = [list(np.nonzero(Mx[j, :])[0]) for j in range(n_sys)]
    Iy = [list(np.nonzero(My[j, :])[0]) for j in range(n_sys)]
    Iz = [list(np.nonzero(Mz[j, :])[0]) for j in range(n_sys)]
    c = {k: [] for k in ("111", "122", "121", "112", "211", "222", "221", "212")}
    c["111"] = [0]

    def gather(I, comps):
        out = []
        for j in comps:
            out.extend(I[j])
        return out

    def total():
        return sum(len(v) for v in c.values())

    guard = 0
    while total() < n_sys:
        c["211"] = sorted(set(c["211"] + gather(Ix, c["111"]) + gather(Iy, c["221"]) + gather(Iz, c["212"])))
        c["121"] = sorted(set(c["121"] + gather(Ix, c["221"]) + gather(Iy, c["111"]) + gather(Iz, c["122"])))
        c["112"] = sorted(set(c["112"] + gather(Ix, c["212"]) + gather(Iy, c["122"]) + gather(Iz, c["111"])))
        c["221"] = sorted(set(c["221"] + gather(Ix, c["121"]) + gather(Iy, c["211"]) + gather(Iz, c["222"])))
        c["212"] = sorted(set(c["212"] + gather(Ix, c["112"]) + gather(Iy, c["222"]) + gather(Iz, c["211"])))
        c["122"] = sorted(set(c["122"] + gather(Ix, c["222"]) + gather(Iy, c["112"]) + gather(Iz, c["121"])))
        c["111"] = sorted(set(c["111"] + gather(Ix, c["211"]) + gather(Iy, c["121"]) + gather(Iz, c["112"])))
        c["222"] = sorted(set(c["222"] + gather(Ix, c["122"]) + gather(Iy, c["212"]) + gather(Iz, c["221"])))
        guard += 1
        if guard > 4 * n_sys + 8:
            raise RuntimeError("grid classification did not converge")
    gtx = np.ones(n_sys, dtype=int)
    gty = np.ones(n_sys, dtype=int)
    gtz = np.ones(n_sys, dtype=int)
    for k in ("211", "212", "221", "222"):
        gtx[c[k]] = 2
    for k in ("121", "122", "221", "222"):
        gty[c[k]] = 2
    for k in ("112", "122", "212", "222"):
        gtz[c[k]] = 2
    return c, Ix, Iy, Iz, gtx, gty, gtz


def starmap_solver(par: dict, *, capture_snapshots: bool = False, max_steps: int | None = None,
                   advance=None, stop=None) -> OracleResult:
    """Run the restated solver.  ``advance`` replaces the numpy step function
    (same arguments as :func:`_advance`); ``oracle.c_oracle`` passes its C one.
    ``max_steps`` or a ``stop()`` callable returning True end the loop early
    (used to time bounded samples)."""
    par = dict(par)
    Mx, My, Mz = (np.asarray(par[k], dtype=np.float64) for k in ("Mx", "My", "Mz"))
    n_sys = Mz.shape[0]
    # flags (starmap_solver.m:58-71)
    if "mom_order" in par:
        f_mom_order = np.atleast_1d(np.asarray(par["mom_order"])).astype(int)
    flag_filter = ("filterfunction" in par) and ("f_position" in par) and ("mom_order" in par)
    if flag_filter:
        f_mom_order = np.atleast_1d(np.asarray(par["mom_order"])).astype(int)
    else:
        par["filterfunction"] = _ones_like_nargin
        par["f_position"] = ""
    flag_ani_scatter = ("sigma_sm" in par) and ("mom_order" in par)
    if not flag_ani_scatter:
        par["mom_order"] = np.concatenate([[0], np.ones(n_sys - 1, dtype=int)])
        par["sigma_sm"] = _zero
    mom_order = np.atleast_1d(np.asarray(par["mom_order"])).astype(int)
    mom_output = par.get("mom_output", 1)
    if isinstance(mom_output, str) and mom_output == "all":
        mom_output = np.arange(1, n_sys + 1)
    mom_output = np.atleast_1d(np.asarray(mom_output)).astype(int)
    f_position = par["f_position"]

    c, Ix, Iy, Iz, gtx, gty, gtz = _classify(Mx, My, Mz)

    # grid size and time step (starmap_solver.m:100-110)
    ax = np.asarray(par["ax"], dtype=np.float64)
    n = np.asarray(par["n"], dtype=int)
    bc = np.asarray(par["bc"], dtype=int)
    h = (ax[[1, 3, 5]] - ax[[0, 2, 4]]) / n
    lam = np.max(np.abs(np.linalg.eigvals(Mz))) if n_sys > 0 else 1.0
    dt_hyp = np.min(h) / abs(lam)
    if n[0] != 1:
        dt_hyp = dt_hyp / 3
    elif n[1] != 1:
        dt_hyp = dt_hyp / 2
    timestep = int(par.get("timestep", 0))
    # von Neumann symbol at the largest wave numbers (starmap_solver.m:108)
    Msym = -1j * (Mx / h[0] + My / h[1] + Mz / h[2])
    time_dependent = np.array([nargin(par["sigma_a"]) > 3, nargin(par["sigma_s0"]) > 3,
                               nargin(par["sigma_sm"]) > 4])

    # staggered grids (starmap_solver.m:112-134)
    xs = [colon(ax[0] + h[0] / 2, h[0], ax[1] - h[0] / 2), colon(ax[0] + h[0] * (1 - bc[0]), h[0], ax[1])]
    ys = [colon(ax[2] + h[1] / 2, h[1], ax[3] - h[1] / 2), colon(ax[2] + h[1] * (1 - bc[1]), h[1], ax[3])]
    zs = [colon(ax[4] + h[2] / 2, h[2], ax[5] - h[2] / 2), colon(ax[4] + h[2] * (1 - bc[2]), h[2], ax[5])]
    X, Y, Z = {}, {}, {}
    for a in (1, 2):
        for b in (1, 2):
            for cz in (1, 2):
                X[a, b, cz], Y[a, b, cz], Z[a, b, cz] = np.meshgrid(xs[a - 1], ys[b - 1], zs[cz - 1], indexing="ij")
    n1 = n
    n2 = np.array(X[2, 2, 2].shape)

    def ext_c2f(nn, b):   # extend{1}: [1:bc, 1:n1, bc*(n1-1)+1]  (0-based)
        return np.array(list(range(0, b)) + list(range(0, nn)) + [b * (nn - 1)], dtype=int)

    def ext_f2c(nn2, b):  # extend{2}: [n2*(1:1-bc), 1:n2]
        return np.array([nn2 - 1] * (1 - b) + list(range(0, nn2)), dtype=int)

    extend = [[ext_c2f(n1[d], bc[d]), ext_f2c(n2[d], bc[d])] for d in range(3)]
    sg_rows = sorted(set((int(gtx[j]), int(gty[j]), int(gtz[j]), int(mom_order[j])) for j in range(1, n_sys)))

    # fields (starmap_solver.m:136-146)
    def G(j):
        return (int(gtx[j]), int(gty[j]), int(gtz[j]))

    ic = par["ic"]
    U = []
    Q = []
    for j in range(n_sys):
        g = G(j)
        val = capargs(ic, X[g], Y[g], Z[g], j + 1)
        U.append(X[g] * 0 + np.asarray(val, dtype=np.float64) * float(nargin(ic) > 3 or j == 0))
        Q.append(X[g] * 0)
    filterTerm = {}
    if flag_filter:
        f_sg_rows = sorted(set((int(gtx[j]), int(gty[j]), int(gtz[j]), int(f_mom_order[j])) for j in range(1, n_sys)))

    # time loop (starmap_solver.m:162-475)
    t_plot = list(np.atleast_1d(np.asarray(par.get("t_plot", [])))) + [np.inf]
    plot_count = 0
    snapshots = []
    t = 0.0
    dt = 0.0
    step_count = 0
    dts = []
    sA = sS = sT = sA0 = sT0 = sA1 = sT1 = None
    sS = {}
    sT = {}
    EA = None
    ET = {}
    tfinal = float(par["tfinal"])
    cn = float(par["cn"])
    source_ind = [int(v) for v in np.atleast_1d(np.asarray(par.get("source_ind", [])))]
    while t < tfinal:
        if max_steps is not None and step_count >= max_steps:
            break
        if stop is not None and stop():
            break
        tleft = (tfinal - t) / cn
        for k in range(int(t > 0), 2):
            if (not time_dependent.any()) and t > 0:
                break
            flag_check_stab = k > 0 and timestep > 0
            if flag_check_stab:
                # parabolic step: bracket and bisect the largest stable dt
                # (starmap_solver.m:173-203)
                dt = max(dt, dt_hyp)
                decay = _decay(sA[1, 1, 1], sT, n_sys, gtx, gty, gtz, mom_order)
                gf = lambda d: _growth_factor(Msym, c, decay, d, timestep)
                la = gf(dt)
                dt_br = [dt, dt]
                la_br = [la, la]
                la0 = 1 + 1e-8
                while ((la_br[0] < la0) == (la_br[1] < la0)) and (dt_br[0] <= tleft or la_br[0] > la0):
                    ind = int(la_br[0] < la0) + 1
                    base = dt_br[ind - 1]
                    dt_br = [base * 1 * 2.0 ** (ind - 2), base * 2 * 2.0 ** (ind - 2)]
                    la_br = [la_br[1], la_br[0]]
                    la_br[ind - 1] = gf(dt_br[ind - 1])
                    if min(la_br) < 1:
                        la0 = 1
                while dt_br[0] / dt_br[1] < 0.98 and dt_br[0] <= tleft:
                    dt_mid = np.sqrt(dt_br[0] * dt_br[1])
                    la_mid = gf(dt_mid)
                    ind = 1 + int(la_mid >= la0)
                    dt_br[ind - 1] = dt_mid
                    la_br[ind - 1] = la_mid
                dt_bracket = dt_br[0]
            else:
                dt_bracket = dt_hyp
            if k > 0:
                dt = min(dt_bracket, tleft) * cn
                sA0 = sA
                sT0 = dict(sT)
                if not time_dependent.any():
                    sA1 = sA[1, 1, 1]
                    sT1 = dict(sT)
                    break
            evaluate = time_dependent | ((dt == 0) & np.array([True, True, flag_ani_scatter]))
            if evaluate[0]:
                sA = {g: np.asarray(capargs(par["sigma_a"], X[g], Y[g], Z[g], t + dt), dtype=np.float64) for g in X}
            if evaluate[1]:
                for (a, b, cz, m) in sg_rows:
                    g = (a, b, cz)
                    sS[a, b, cz, m] = np.asarray(capargs(par["sigma_s0"], X[g], Y[g], Z[g], t + dt), dtype=np.float64)
            if evaluate[2]:
                for (a, b, cz, m) in sg_rows:
                    g = (a, b, cz)
                    sS[a, b, cz, m] = sS[a, b, cz, m] - np.asarray(
                        capargs(par["sigma_sm"], X[g], Y[g], Z[g], m, t + dt), dtype=np.float64)
            if evaluate.any():
                for (a, b, cz, m) in sg_rows:
                    sT[a, b, cz, m] = sA[a, b, cz] + sS[a, b, cz, m]
            if k > 0:
                sA1 = (sA0[1, 1, 1] + sA[1, 1, 1]) / 2
                sT1 = {key: (sT0[key] + sT[key]) / 2 for key in sg_rows}
            if flag_check_stab:
                # averaged materials unstable with dt: fall back to those at t
                # (starmap_solver.m:253-265)
                decay = _decay(sA1, sT1, n_sys, gtx, gty, gtz, mom_order)
                if not _growth_factor(Msym, c, decay, dt, timestep) < la0:
                    sA1 = sA0[1, 1, 1]
                    sT1 = sT0
        # decay terms (starmap_solver.m:267-274)
        if t == 0 or time_dependent.any():
            EA = expm1div(-sA1 * dt / 2)
            for key in sg_rows:
                ET[key] = expm1div(-sT1[key] * dt / 2)
        t = t + dt
        dts.append(dt)
        step_count += 1
        for j1 in source_ind:
            j = j1 - 1
            g = G(j)
            Q[j] = np.asarray(capargs(par["source"], X[g], Y[g], Z[g], t - dt / 2, j1), dtype=np.float64)
        if (t == dt or nargin(par["filterfunction"]) > 6) and flag_filter:
            for (a, b, cz, m) in f_sg_rows:
                g = (a, b, cz)
                if f_position == "full":
                    filterTerm[a, b, cz, m] = np.asarray(capargs(par["filterfunction"], par, dt, m, X[g], Y[g], Z[g], t), dtype=np.float64)
                elif f_position == "substep":
                    filterTerm[a, b, cz, m, 1] = np.asarray(capargs(par["filterfunction"], par, dt, m, X[g], Y[g], Z[g], t - dt / 2), dtype=np.float64)
                    filterTerm[a, b, cz, m, 2] = np.asarray(capargs(par["filterfunction"], par, dt, m, X[g], Y[g], Z[g], t), dtype=np.float64)
        U0 = [U[j - 1] for j in mom_output]
        (advance or _advance)(U, Q, Ix, Iy, Iz, c, extend, h, Mx, My, Mz, dt, gtx, gty, gtz, mom_order, f_mom_order if flag_filter else None,
                 f_position, sA1, EA, sT1, ET, filterTerm)
        # plotting/interpolation (starmap_solver.m:425-473), headless
        while t >= t_plot[plot_count] - 1e-14:
            lam_p = (t_plot[plot_count] - t + dt) / dt
            Uplot = [(1 - lam_p) * u0 + lam_p * U[j - 1] for u0, j in zip(U0, mom_output)]
            if capture_snapshots:
                snapshots.append((t_plot[plot_count], Uplot))
            plot_count += 1
    # output (starmap_solver.m:484-500)
    dim = par.get("dim", 3)
    out = []
    for j in range(n_sys):
        if dim == 1:
            out.append({"x": zs[gtz[j] - 1], "U": U[j].reshape(len(zs[gtz[j] - 1]), -1, order="F")})
        elif dim == 2:
            out.append({"x": ys[gty[j] - 1], "y": zs[gtz[j] - 1],
                        "U": U[j].reshape(len(ys[gty[j] - 1]), -1, order="F")})
        else:
            out.append({"x": xs[gtx[j] - 1], "y": ys[gty[j] - 1], "z": zs[gtz[j] - 1], "U": U[j]})
    setup = dict(c=c, gtx=gtx, gty=gty, gtz=gtz, h=h, dt_hyp=dt_hyp, EA=EA, ET=ET, sA1=sA1, sT1=sT1,
                 filterTerm=filterTerm, Q=Q, mom_order=mom_order)
    return OracleResult(out, U, step_count, t, dt, snapshots, setup, dts)


def _advance(U, Q, Ix, Iy, Iz, c, extend, h, Mx, My, Mz, dt, gtx, gty, gtz, mom_order, f_mom_order, f_position,
             sA1, EA, sT1, ET, filterTerm):
    """One Strang-split step A-B-A plus the full filter (starmap_solver.m:309-421)."""
    n_sys = len(U)
    dU = [dict() for _ in range(n_sys)]   # dU[j][d] = derivative along solver dim d

    def deriv(j, g):
        # g: grid-type triple of comp j (1 = centre, 2 = staggered)
        if Ix[j]:
            dU[j][0] = np.diff(U[j][extend[0][g[0] - 1], :, :], axis=0) / h[0]
        if Iy[j]:
            dU[j][1] = np.diff(U[j][:, extend[1][g[1] - 1], :], axis=1) / h[1]
        dU[j][2] = np.diff(U[j][:, :, extend[2][g[2] - 1]], axis=2) / h[2]

    def W_of(j):
        terms = [(dU[i][0], Mx[j, i]) for i in Ix[j]] + [(dU[i][1], My[j, i]) for i in Iy[j]] + \
                [(dU[i][2], Mz[j, i]) for i in Iz[j]]
        S = terms[0][0] * terms[0][1]
        for A, w in terms[1:]:
            S = S + A * w
        return -S

    def key(j):
        return (int(gtx[j]), int(gty[j]), int(gtz[j]), int(mom_order[j]))

    def fkey(j):
        return (int(gtx[j]), int(gty[j]), int(gtz[j]), int(f_mom_order[j]))

    k = 1
    for step in (1, 2, 1):
        if step == 1:
            for cls, g in (("111", (1, 1, 1)), ("221", (2, 2, 1)), ("212", (2, 1, 2)), ("122", (1, 2, 2))):
                for j in c[cls]:
                    deriv(j, g)
            for j in c["211"] + c["121"] + c["112"] + c["222"]:
                W = W_of(j)
                U[j] = U[j] + dt / 2 * (W + Q[j] - sT1[key(j)] * U[j]) * ET[key(j)]
                if f_position == "substep":
                    U[j] = U[j] * filterTerm[fkey(j) + (k,)]
        else:
            for cls, g in (("222", (2, 2, 2)), ("112", (1, 1, 2)), ("121", (1, 2, 1)), ("211", (2, 1, 1))):
                for j in c[cls]:
                    deriv(j, g)
            for j in c["111"] + c["221"] + c["212"] + c["122"]:
                W = W_of(j)
                for k in (1, 2):
                    if j == 0:
                        U[j] = U[j] + dt / 2 * (W + Q[j] - sA1 * U[j]) * EA
                    else:
                        U[j] = U[j] + dt / 2 * (W + Q[j] - sT1[key(j)] * U[j]) * ET[key(j)]
                        if f_position == "substep":
                            U[j] = U[j] * filterTerm[fkey(j) + (k,)]
    if f_position == "full":
        for j in range(1, n_sys):
            U[j] = U[j] * filterTerm[fkey(j)]

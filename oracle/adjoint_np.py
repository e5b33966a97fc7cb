"""CPU discrete adjoint of the restated time loop (numpy, FP64).

TEST INFRASTRUCTURE ONLY: the checker for the GPU adjoint (smg_forward /
smg_backward).  Only tests may import it; the library never does.

The reference has no derivatives; what is differentiated is exactly the
restated loop of ``oracle/solver_np.py`` (``_advance``, which follows
starmap_solver.m:309-421): per step phase A with filter k=1, phase B (two
substeps sharing one coupling sum W), phase A with filter k=2.  For each
destination j of a phase

    u' = F * (u + (dt/2) * (W + q - s*u) * E),   E = expm1div(-s*dt/2),
    W  = -sum_i M_d(j,i) * D_d U_i,   D_d U = diff(U(ext_d), d) / h_d

(starmap_solver.m:350-357, 398-411, 127-132).  The backward sweep stores the
state before every phase and every W, then runs the phases in reverse:

    lambda_j <- F (1 - (dt/2) s E) lambda'_j            (pointwise part)
    v_j       = F (dt/2) E lambda'_j                     (dJ/dW_j)
    dJ/ds    += F (dt/2) (-u E + (W + q - s u) dE/ds) lambda'_j
    dJ/dq    += v_j
    lambda_i += -sum_j M_d(j,i) D_d^T v_j                (sources i)

with D_d^T scattering +v/h onto ext[p+1] and -v/h onto ext[p] (np.add.at).
Decay factors are functions of sigma (their derivative enters dJ/dsigma);
filters are constants.  Autonomous problems with f_position '' or 'substep'.
"""
from __future__ import annotations

import numpy as np

from . import solver_np as O


def dexpm1div(x):
    """d/dx of expm1div with the reference's Taylor branch (starmap_solver.m:531-535):
    1/2 + x/3 where |x| <= 2e-4, the series sum_k k x^(k-1)/(k+1)! for |x| < 0.25,
    (x e^x - e^x + 1)/x^2 otherwise."""
    x = np.asarray(x, dtype=np.float64)
    out = np.empty_like(x)
    small = np.abs(x) <= 2e-4
    mid = (~small) & (np.abs(x) < 0.25)
    big = ~(small | mid)
    out[small] = 0.5 + x[small] / 3.0
    xm = x[mid]
    acc = np.zeros_like(xm)
    fact = 2.0          # (k+1)! for k = 1
    xp = np.ones_like(xm)
    for k in range(1, 18):
        acc = acc + k * xp / fact
        xp = xp * xm
        fact = fact * (k + 2)
    out[mid] = acc
    xb = x[big]
    out[big] = (xb * np.exp(xb) - np.exp(xb) + 1.0) / (xb * xb)
    return out


def _diffT(v, ext, axis, h, shape):
    """Adjoint of U -> diff(U(ext), axis)/h: scatter v/h onto ext[p+1] and -v/h onto ext[p]."""
    acc = np.zeros(shape)
    t = np.moveaxis(v / h, axis, 0)
    a = np.moveaxis(acc, axis, 0)
    ext = np.asarray(ext)
    np.add.at(a, ext[1:], t)
    np.add.at(a, ext[:-1], -t)
    return acc


class _Recorder:
    """An ``advance`` for the oracle loop that performs ``_advance``'s step
    (same operations and order) and records what the backward sweep needs."""

    def __init__(self, U0=None):
        self.phases = []     # per phase: dict
        self.steps = 0
        self.U0 = U0         # optional initial state replacing the sampled one

    def __call__(self, U, Q, Ix, Iy, Iz, c, extend, h, Mx, My, Mz, dt, gtx, gty, gtz, mom_order, f_mom_order,
                 f_position, sA1, EA, sT1, ET, filterTerm):
        if f_position == "full":
            raise NotImplementedError("the adjoint covers f_position '' and 'substep'")
        n_sys = len(U)
        if self.steps == 0 and self.U0 is not None:
            for j in range(n_sys):
                U[j] = np.array(self.U0[j], dtype=np.float64).reshape(U[j].shape)
        self.ctx = dict(Ix=Ix, Iy=Iy, Iz=Iz, extend=extend, h=h, M=(Mx, My, Mz), dt=dt,
                        gt=(gtx, gty, gtz), mom_order=mom_order, f_mom_order=f_mom_order, f_position=f_position,
                        sA1=sA1, EA=EA, sT1=sT1, ET=ET, filterTerm=filterTerm, Q=Q, n_sys=n_sys)
        key = lambda j: (int(gtx[j]), int(gty[j]), int(gtz[j]), int(mom_order[j]))
        fkey = lambda j: (int(gtx[j]), int(gty[j]), int(gtz[j]), int(f_mom_order[j]))
        hdt = dt / 2
        k = 1
        for step in (1, 2, 1):
            if step == 1:
                src = [("111", (1, 1, 1)), ("221", (2, 2, 1)), ("212", (2, 1, 2)), ("122", (1, 2, 2))]
                dst = c["211"] + c["121"] + c["112"] + c["222"]
            else:
                src = [("222", (2, 2, 2)), ("112", (1, 1, 2)), ("121", (1, 2, 1)), ("211", (2, 1, 1))]
                dst = c["111"] + c["221"] + c["212"] + c["122"]
            gsrc = {}
            dU = [dict() for _ in range(n_sys)]
            for cls, g in src:
                for j in c[cls]:
                    gsrc[j] = g
                    if Ix[j]:
                        dU[j][0] = np.diff(U[j][extend[0][g[0] - 1], :, :], axis=0) / h[0]
                    if Iy[j]:
                        dU[j][1] = np.diff(U[j][:, extend[1][g[1] - 1], :], axis=1) / h[1]
                    dU[j][2] = np.diff(U[j][:, :, extend[2][g[2] - 1]], axis=2) / h[2]
            rec = dict(step=step, k=k, dests=[], gsrc=gsrc)
            for j in dst:
                terms = [(dU[i][0], Mx[j, i]) for i in Ix[j]] + [(dU[i][1], My[j, i]) for i in Iy[j]] + \
                        [(dU[i][2], Mz[j, i]) for i in Iz[j]]
                S = terms[0][0] * terms[0][1]
                for A, w in terms[1:]:
                    S = S + A * w
                W = -S
                if step == 1:
                    s, E = sT1[key(j)], ET[key(j)]
                    F = filterTerm[fkey(j) + (k,)] if f_position == "substep" else 1.0
                    u = U[j]
                    U[j] = U[j] + hdt * (W + Q[j] - s * U[j]) * E
                    if f_position == "substep":
                        U[j] = U[j] * F
                    rec["dests"].append(dict(j=j, u=u, W=W, s=s, E=E, F=(F,), key=key(j)))
                else:
                    u = U[j]
                    mids = []
                    Fs = []
                    for k in (1, 2):
                        mids.append(U[j])
                        if j == 0:
                            s, E, F = sA1, EA, 1.0
                            U[j] = U[j] + hdt * (W + Q[j] - s * U[j]) * E
                        else:
                            s, E = sT1[key(j)], ET[key(j)]
                            F = filterTerm[fkey(j) + (k,)] if f_position == "substep" else 1.0
                            U[j] = U[j] + hdt * (W + Q[j] - s * U[j]) * E
                            if f_position == "substep":
                                U[j] = U[j] * F
                        Fs.append(F)
                    rec["dests"].append(dict(j=j, u=mids, W=W, s=s, E=E, F=tuple(Fs),
                                             key=None if j == 0 else key(j)))
            self.phases.append(rec)
        self.steps += 1


def adjoint(par: dict, nsteps: int, seed, U0=None):
    """Forward ``nsteps`` steps of the restated loop from ``par``'s initial
    condition (or from ``U0``, a list per component), then the adjoint sweep.  ``seed(U_final)`` returns the adjoint
    of the final state (list per component) and optionally a misfit value, as
    ``(lam, J)``.  Returns dict with ``U`` (final state), ``J``, ``lam0``
    (dJ/dU(0) per component), ``g_sT`` ({(g1,g2,g3,m): array or float}),
    ``g_sA`` (array or float), ``g_Q`` ({component: array or float})."""
    rec = _Recorder(U0)
    res = O.starmap_solver(par, max_steps=nsteps, advance=rec)
    if rec.steps != nsteps:
        raise ValueError(f"the loop ended after {rec.steps} steps (tfinal reached), fewer than {nsteps}")
    U = res.U
    lam, J = seed(U)
    lam = [np.array(l, dtype=np.float64, copy=True).reshape(U[j].shape) for j, l in enumerate(lam)]
    ctx = rec.ctx
    hdt = ctx["dt"] / 2
    extend, h = ctx["extend"], ctx["h"]
    Ix, Iy, Iz = ctx["Ix"], ctx["Iy"], ctx["Iz"]
    Mx, My, Mz = ctx["M"]
    g_s = {}            # key -> per-point accumulation (sT fields)
    g_a = 0.0           # sA1
    g_q = {}

    def dE_of(s):
        return -hdt * dexpm1div(-np.asarray(s, dtype=np.float64) * hdt)

    def add(d, k, v):
        d[k] = d[k] + v if k in d else v

    for ph in reversed(rec.phases):
        V = {}
        for d in ph["dests"]:
            j = d["j"]
            lp = lam[j]
            s, E, W = d["s"], d["E"], d["W"]
            q = ctx["Q"][j]
            dE = dE_of(s)
            r = 1.0 - hdt * s * E
            if ph["step"] == 1:
                F = d["F"][0]
                u = d["u"]
                lam[j] = F * r * lp
                v = F * hdt * E * lp
                gs = F * hdt * (-u * E + (W + q - s * u) * dE) * lp
            else:
                F1, F2 = d["F"]
                u0, u1 = d["u"]
                l1 = F2 * r * lp
                v = F2 * hdt * E * lp
                gs = F2 * hdt * (-u1 * E + (W + q - s * u1) * dE) * lp
                lam[j] = F1 * r * l1
                v = v + F1 * hdt * E * l1
                gs = gs + F1 * hdt * (-u0 * E + (W + q - s * u0) * dE) * l1
            V[j] = v
            if j == 0 and ph["step"] == 2:
                g_a = g_a + gs
            else:
                add(g_s, d["key"], gs)
            add(g_q, j, v)
        # transposed coupling onto the sources of the phase
        for d in ph["dests"]:
            j = d["j"]
            v = V[j]
            for lst, M, ax in ((Ix[j], Mx, 0), (Iy[j], My, 1), (Iz[j], Mz, 2)):
                for i in lst:
                    g = ph["gsrc"][i]
                    lam[i] = lam[i] - M[j, i] * _diffT(v, extend[ax][g[ax] - 1], ax, h[ax], lam[i].shape)

    def fold(field, acc):
        # a scalar coefficient gets the sum over the points it acts on
        return float(np.sum(acc)) if np.ndim(field) == 0 else acc

    g_sT = {k: fold(ctx["sT1"][k], v) for k, v in g_s.items()}
    g_sA = fold(ctx["sA1"], g_a)
    g_Q = {j: fold(ctx["Q"][j], v) for j, v in g_q.items() if np.ndim(ctx["Q"][j]) > 0 or ctx["Q"][j] != 0}
    return dict(U=U, J=J, lam0=lam, g_sT=g_sT, g_sA=g_sA, g_Q=g_Q, steps=rec.steps)


def misfit_seed(obs):
    """Seed of J = 1/2 sum (U_1(T) - obs)^2 (zeroth moment)."""
    def seed(U):
        r = U[0] - np.asarray(obs, dtype=np.float64).reshape(U[0].shape)
        lam = [r] + [np.zeros_like(u) for u in U[1:]]
        return lam, 0.5 * float(np.sum(r * r))
    return seed

"""Algorithmic HBM bytes of the time loop (the roofline numerator).

Per phase of the Strang step the minimum traffic of the fused-phase design is:
every component read once (sources for the differences, destinations for the
update), every destination written once, and each distinct coefficient array
(sigma_t / decay / source / filter fields) read once.  A step is phase A,
phase B, phase A (starmap_solver.m:310), plus the full filter pass when
``f_position == 'full'`` (starmap_solver.m:417-421).
"""
from __future__ import annotations

import numpy as np


def _points(S, grid):
    return int(np.prod([(S.n[d] + 1) if (grid[d] == 2 and S.bc[d] == 1) else S.n[d] for d in range(3)]))


def algorithmic_bytes_per_step(S, T, fused: bool = False) -> dict:
    """Bytes per step for setup ``S`` and field table ``T`` (see solver.setup_gpu).

    ``fused``: phase A at the end of a step and at the start of the next run as
    one pass (the library's default), so a step in the middle of a run costs one
    phase-A pass (with both filter terms) and one phase-B pass."""
    n_sys = S.n_sys
    pts = [_points(S, S.G(j)) for j in range(n_sys)]
    outer = [j for j in range(n_sys) if sum(g == 2 for g in S.G(j)) % 2 == 1]
    inner = [j for j in range(n_sys) if j not in set(outer)]
    fields = T.fields

    def is_array(k):
        return k is not None and np.ndim(fields[k][0]) > 0

    def fsize(k):
        return _points(S, fields[k][1])

    def phase(dests, which):
        used = set()
        for j in dests:
            if j == 0:
                used.update([T.index[("sA",)], T.index[("EA",)]])
            else:
                key = (*S.G(j), int(S.mom_order[j]))
                used.update([T.index[("sT",) + key], T.index[("ET",) + key]])
            q = T.index.get(("Q", j))
            if q is not None:
                used.add(q)
            if S.flag_filter and S.f_position == "substep" and j > 0:
                fk = (*S.G(j), int(S.f_mom_order[j]))
                for k in which:
                    used.add(T.index[("F",) + fk + (k,)])
        arr = sum(fsize(k) for k in used if is_array(k))
        return 8 * (sum(pts) + sum(pts[j] for j in dests) + arr)

    A1 = phase(outer, (1,))
    B = phase(inner, (1, 2))
    A2 = phase(outer, (2,))
    if fused and not (S.flag_filter and S.f_position == "full"):
        AA = phase(outer, (1, 2))
        state = 8 * sum(pts)
        return dict(phase_AA=AA, phase_B=B, full_filter=0, step=AA + B, state_bytes=state,
                    n_outer=len(outer), n_inner=len(inner), fused=True)
    full = 0
    if S.flag_filter and S.f_position == "full":
        used = {T.index[("F", *S.G(j), int(S.f_mom_order[j]))] for j in range(1, n_sys)}
        full = 8 * (2 * sum(pts[1:]) + sum(fsize(k) for k in used if is_array(k)))
    state = 8 * sum(pts)
    return dict(phase_A=A1, phase_B=B, phase_A2=A2, full_filter=full, step=A1 + B + A2 + full,
                state_bytes=state, n_outer=len(outer), n_inner=len(inner))

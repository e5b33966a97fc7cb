"""Many StaRMAP problems advanced together on one GPU (``smg_batch_*``).

A batch replaces a host loop of ``starmap_solver`` calls: every instance keeps
its own grid, moment order, coefficients and dt, and all of them are stepped
by one persistent launch per block of steps (see starmap_b200/csrc/smg_batch.cu).
"""
from __future__ import annotations

import numpy as np

from . import _lib
from ._lib import check_batch
from .solver import GpuSolver, build_problem, first_step, handle_tables, prepare, _Tables

__all__ = ["GpuBatch", "setup_batch"]

BLOCK, GROUP, STEPS_PER_LAUNCH, SPIN_LIMIT, BARRIER_EXTRA, USE_GRAPH, PERSISTENT, JIT = 1, 2, 3, 4, 5, 6, 7, 8


def _tables(S, fs):
    T = _Tables()
    for row in S.sg:
        T.add(("sT",) + row, fs["sT1"][row], row[:3])
        T.add(("ET",) + row, fs["ET"][row], row[:3])
    T.add(("sA",), fs["sA1"], (1, 1, 1))
    T.add(("EA",), fs["EA"], (1, 1, 1))
    for j, q in fs["Q"].items():
        T.add(("Q", j), q, S.G(j))
    for key, val in fs["F"].items():
        T.add(("F",) + key, val, key[:3])
    return T


class GpuBatch:
    """Owner of one ``smg_batch``."""

    def __init__(self, setups):
        """``setups``: list of (S, fs) from :func:`prepare` / :func:`first_step`."""
        L = _lib.lib()
        self._L = L
        probs, keeps, self.infos = [], [], []
        self.S = [S for S, _ in setups]
        self.dt = [fs["dt"] for _, fs in setups]
        for S, fs in setups:
            T = _tables(S, fs)
            p, keep, info = build_problem(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, T.fields, **handle_tables(S, T))
            probs.append(p)
            keeps.append(keep)
            self.infos.append(info)
        arr = (_lib.C.POINTER(_lib.smg_problem) * len(probs))(*[_lib.C.pointer(p) for p in probs])
        b = _lib.C.c_void_p()
        check_batch(L.smg_batch_create(len(probs), arr, _lib.C.byref(b)))
        self.b = b
        self.n = len(probs)
        self.inst = [GpuSolver.borrow(L.smg_batch_instance(b, i), self.infos[i]) for i in range(self.n)]

    def set_states(self, U_list):
        for solver, U in zip(self.inst, U_list):
            solver.set_state(U)

    def set_dt(self, dts):
        a = np.ascontiguousarray(np.asarray(dts, dtype=np.float64))
        check_batch(self._L.smg_batch_set_dt(self.b, _lib.dptr(a)), self.b)

    def run(self, nsteps):
        check_batch(self._L.smg_batch_run(self.b, int(nsteps)), self.b)

    def tune(self, key, value):
        check_batch(self._L.smg_batch_tune(self.b, int(key), int(value)), self.b)

    def info(self):
        """(generated family kernels used by the last runs, number of families)."""
        j = _lib.C.c_int64()
        f = _lib.C.c_int64()
        check_batch(self._L.smg_batch_info(self.b, _lib.C.byref(j), _lib.C.byref(f)), self.b)
        return bool(j.value), f.value

    def config(self):
        out = (_lib.C.c_int64 * 4)()
        check_batch(self._L.smg_batch_config(self.b, out), self.b)
        return dict(block=out[0], group=out[1], steps_per_launch=out[2], grid=out[3])

    def autotune(self, probe_steps=4):
        ms = _lib.C.c_double()
        check_batch(self._L.smg_batch_autotune(self.b, int(probe_steps), _lib.C.byref(ms)), self.b)
        return ms.value

    def last_run_stats(self):
        ms = _lib.C.c_double()
        nl = _lib.C.c_int64()
        check_batch(self._L.smg_batch_last_run_stats(self.b, _lib.C.byref(ms), _lib.C.byref(nl)), self.b)
        return ms.value, nl.value

    def get_state(self, i, which=None):
        return self.inst[i].get_state(which)

    def close(self):
        if getattr(self, "b", None):
            for s in self.inst:
                s.h = None
            self._L.smg_batch_destroy(self.b)
            self.b = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def setup_batch(pars):
    """Host setup of every ``par`` and the batch handle (states/dt not yet set).

    A batch advances every instance with the coefficients of its first step
    and a fixed dt, so it takes autonomous problems only: materials, sources
    and filters whose hooks depend on t are refused (they need the per-step
    path of ``starmap_solver``, starmap_solver.m:165-305)."""
    setups = []
    for i, par in enumerate(pars):
        S = prepare(par)
        if S.time_dependent.any() or S.src_td or S.filter_td:
            raise ValueError(f"batch instance {i}: time-dependent materials, sources or filters are not "
                             "supported by the batched solver (run it through starmap_solver)")
        setups.append((S, first_step(S)))
    return setups, GpuBatch(setups)

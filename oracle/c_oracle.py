"""ORACLE (test infrastructure only) -- ctypes driver of oracle/loop_ref.c.

``CAdvance`` is a drop-in for the numpy step function of
``oracle.solver_np.starmap_solver`` (its ``advance=`` argument): the numpy
restatement keeps doing the setup and the per-step hook evaluation, and each
Strang step is executed by the C restatement in place on the same component
arrays.  Use ``run(par, nthreads)`` for a full solve.
"""
from __future__ import annotations

import ctypes as C
import time

import numpy as np

from . import build as _build
from . import solver_np

_lib = None


class ofield(C.Structure):
    _fields_ = [("p", C.POINTER(C.c_double)), ("s", C.c_double)]


class oracle_desc(C.Structure):
    _fields_ = [
        ("n_sys", C.c_int32), ("n", C.c_int32 * 3), ("bc", C.c_int32 * 3), ("h", C.c_double * 3),
        ("hdt", C.c_double), ("filter_mode", C.c_int32),
        ("ext", C.POINTER(C.c_int32)), ("gt", C.POINTER(C.c_int32)),
        ("cptr", C.POINTER(C.c_int32)), ("csrc", C.POINTER(C.c_int32)), ("cdir", C.POINTER(C.c_int32)),
        ("cw", C.POINTER(C.c_double)),
        ("destA", C.POINTER(C.c_int32)), ("nA", C.c_int32),
        ("destB", C.POINTER(C.c_int32)), ("nB", C.c_int32),
        ("sT", C.POINTER(ofield)), ("ET", C.POINTER(ofield)), ("Q", C.POINTER(ofield)),
        ("F1", C.POINTER(ofield)), ("F2", C.POINTER(ofield)),
        ("sA1", ofield), ("EA", ofield),
    ]


def lib():
    global _lib
    if _lib is None:
        path = _build.build()
        L = C.CDLL(path)
        L.oracle_step.restype = C.c_int
        L.oracle_step.argtypes = [C.POINTER(oracle_desc), C.POINTER(C.POINTER(C.c_double)), C.c_int]
        L.oracle_max_threads.restype = C.c_int
        _lib = L
    return _lib


def _i32(a):
    return np.ascontiguousarray(np.asarray(a, dtype=np.int32))


class CAdvance:
    """Stateful step function; see module docstring."""

    def __init__(self, nthreads: int = 0):
        self.nthreads = int(nthreads)
        self.static = None
        self.cache = {}
        self.step_seconds = []   # wall time of each C step (kernel of the CPU baseline)

    def _field(self, val, shape):
        if val is None:
            return ofield(None, 0.0), None
        a = np.asarray(val)
        if a.ndim == 0:
            return ofield(None, float(a)), None
        key = (id(val), shape)
        hit = self.cache.get(key)
        if hit is None or hit[0] is not val:
            arr = np.asfortranarray(np.broadcast_to(a.astype(np.float64, copy=False), shape))
            hit = (val, arr)
            self.cache[key] = hit
        arr = hit[1]
        return ofield(arr.ctypes.data_as(C.POINTER(C.c_double)), 0.0), arr

    def __call__(self, U, Q, Ix, Iy, Iz, c, extend, h, Mx, My, Mz, dt, gtx, gty, gtz, mom_order,
                 f_mom_order, f_position, sA1, EA, sT1, ET, filterTerm):
        n_sys = len(U)
        if self.static is None:
            ext = np.array([U[j].shape for j in range(n_sys)], dtype=np.int32)
            cptr, csrc, cdir, cw = [0], [], [], []
            for j in range(n_sys):
                for d, (I, M) in enumerate(((Ix, Mx), (Iy, My), (Iz, Mz))):
                    for i in I[j]:
                        csrc.append(i)
                        cdir.append(d)
                        cw.append(M[j, i])
                cptr.append(len(csrc))
            destA = c["211"] + c["121"] + c["112"] + c["222"]
            destB = c["111"] + c["221"] + c["212"] + c["122"]
            self.static = dict(ext=_i32(ext.ravel()), gt=_i32(np.stack([gtx, gty, gtz], 1).ravel()),
                               cptr=_i32(cptr), csrc=_i32(csrc), cdir=_i32(cdir),
                               cw=np.ascontiguousarray(np.asarray(cw, dtype=np.float64)),
                               destA=_i32(destA), destB=_i32(destB), ext_shape=[tuple(e) for e in ext])
        st = self.static
        for j in range(n_sys):
            if not (U[j].flags.f_contiguous and U[j].dtype == np.float64):
                U[j] = np.asfortranarray(U[j], dtype=np.float64)
        keep = []
        mode = {"": 0, "substep": 1, "full": 2}.get(f_position, 0)
        if f_mom_order is None:
            mode = 0
        sT = (ofield * n_sys)()
        Et = (ofield * n_sys)()
        Qf = (ofield * n_sys)()
        F1 = (ofield * n_sys)()
        F2 = (ofield * n_sys)()
        for j in range(n_sys):
            shape = st["ext_shape"][j]
            g = (int(gtx[j]), int(gty[j]), int(gtz[j]))
            if j > 0:
                key = g + (int(mom_order[j]),)
                sT[j], a = self._field(sT1[key], shape); keep.append(a)
                Et[j], a = self._field(ET[key], shape); keep.append(a)
            Qf[j], a = self._field(Q[j], shape); keep.append(a)
            F1[j] = ofield(None, 1.0)
            F2[j] = ofield(None, 1.0)
            if mode and j > 0:
                fk = g + (int(f_mom_order[j]),)
                if mode == 1:
                    F1[j], a = self._field(filterTerm[fk + (1,)], shape); keep.append(a)
                    F2[j], a = self._field(filterTerm[fk + (2,)], shape); keep.append(a)
                else:
                    F1[j], a = self._field(filterTerm[fk], shape); keep.append(a)
        d = oracle_desc()
        d.n_sys = n_sys
        d.n[:] = [len(extend[k][1]) - 1 for k in range(3)]   # extend{2} has n+1 entries
        d.bc[:] = [int(len(extend[k][0]) - len(extend[k][1]) == 1) for k in range(3)]
        d.h[:] = [float(v) for v in h]
        d.hdt = dt / 2
        d.filter_mode = mode
        P = lambda a, t=C.c_int32: a.ctypes.data_as(C.POINTER(t))
        d.ext, d.gt, d.cptr, d.csrc, d.cdir = P(st["ext"]), P(st["gt"]), P(st["cptr"]), P(st["csrc"]), P(st["cdir"])
        d.cw = P(st["cw"], C.c_double)
        d.destA, d.nA = P(st["destA"]), len(st["destA"])
        d.destB, d.nB = P(st["destB"]), len(st["destB"])
        d.sT, d.ET, d.Q, d.F1, d.F2 = sT, Et, Qf, F1, F2
        d.sA1, a = self._field(sA1, st["ext_shape"][0]); keep.append(a)
        d.EA, a = self._field(EA, st["ext_shape"][0]); keep.append(a)
        ptrs = (C.POINTER(C.c_double) * n_sys)(*[U[j].ctypes.data_as(C.POINTER(C.c_double)) for j in range(n_sys)])
        t0 = time.perf_counter()
        lib().oracle_step(C.byref(d), ptrs, self.nthreads)
        self.step_seconds.append(time.perf_counter() - t0)


def run(par, nthreads: int = 0, max_steps=None, capture_snapshots=False, advance=None, stop=None):
    """Full solve: numpy setup + C steps (pass ``advance`` to read its step timings)."""
    return solver_np.starmap_solver(par, advance=advance or CAdvance(nthreads), max_steps=max_steps,
                                    capture_snapshots=capture_snapshots, stop=stop)


def max_threads() -> int:
    return int(lib().oracle_max_threads())

"""``output = starmap_solver(par)`` on the GPU.

Host side of the drop-in for StaRMAP's ``starmap_solver.m``.  The setup that
the reference performs before its update loop stays on the host and follows
the reference statement by statement (flags :58-71, grid-type classification
:76-98 -- computed by the library's ``smg_classify`` --, h and dt :100-110,
staggered grids :112-134, initial and source fields :136-146, materials, dt,
decay factors, source and filter tables at the first step :165-305).  The time
loop itself (:307-421) runs in ``libstarmap_gpu.so`` through the C ABI of
``include/starmap_gpu.h``; the final components come back in the reference's
``output`` layout (:484-500) and the reference's summary is printed (:477-482).

Autonomous problems run the whole loop in one library call (replayed CUDA
graphs for light steps, direct launches for heavy ones).  Time-dependent materials, sources or filters are re-evaluated on the
host every step exactly where the reference does, uploaded with
``smg_set_field`` and advanced one step at a time.  Output times ``t_plot``
with a user ``output`` hook are served by running the loop in segments and
interpolating linearly in time as the reference does (:425-473).
"""
from __future__ import annotations

import math
import re
import time

import numpy as np

from . import _lib
from ._lib import FILTER_FULL, FILTER_NONE, FILTER_SUBSTEP, check, dptr, iptr
from . import timestep
from .init import _noop_output, capargs, nargin, zero

__all__ = ["starmap_solver", "GpuSolver", "prepare", "expm1div", "colon", "step_times"]

VARIANT_AUTO, VARIANT_GENERIC, VARIANT_STRIP = 0, 1, 2
#: kernel family used by :func:`starmap_solver` (all variants give identical results)
DEFAULT_VARIANT = VARIANT_AUTO


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
    """Octave range ``a:d:b``: base + k*increment, last element clamped to the limit."""
    n = int(math.floor((b - a) / d + 1e-10)) + 1
    if n <= 0:
        return np.zeros(0)
    v = a + np.arange(n) * d
    if n > 1:
        v[-1] = min(a + (n - 1) * d, b)
    return v


def step_times(dt: float, tfinal: float):
    """Times after each step of the autonomous loop (starmap_solver.m:165, 276).

    dt is fixed after the first step, so the loop overshoots tfinal."""
    ts = []
    t = 0.0
    while t < tfinal:
        t = t + dt
        ts.append(t)
    return ts


class GpuSolver:
    """Owner of one ``smg_handle``: the problem on the GPU."""

    def __init__(self, n, bc, h, gt, Mx, My, Mz, fields, sigma_t, sigma_a, source,
                 decay_t=None, decay_a=-1, filter_mode=FILTER_NONE, filter1=None, filter2=None):
        L = _lib.lib()
        self._L = L
        self.field_scalar = [np.ndim(v) == 0 for v, _ in fields]
        p, keep, info = build_problem(n, bc, h, gt, Mx, My, Mz, fields, sigma_t, sigma_a, source,
                                      decay_t, decay_a, filter_mode, filter1, filter2)
        self.n_sys, self.n, self.bc, self.gt, self.field_grids = info
        handle = _lib.C.c_void_p()
        check(L.smg_create(_lib.C.byref(p), _lib.C.byref(handle)))
        self.h = handle
        self.owned = True

    @classmethod
    def borrow(cls, handle, info):
        """Wrap a handle owned by someone else (a batch instance)."""
        self = cls.__new__(cls)
        self._L = _lib.lib()
        self.n_sys, self.n, self.bc, self.gt, self.field_grids = info
        self.h = handle
        self.owned = False
        return self

    # ------------------------------------------------------------------
    def extents(self, j):
        return tuple((self.n[d] + 1) if (self.gt[j, d] == 2 and self.bc[d] == 1) else self.n[d] for d in range(3))

    def grid_extents(self, grid):
        return tuple((self.n[d] + 1) if (grid[d] == 2 and self.bc[d] == 1) else self.n[d] for d in range(3))

    def _extents_all(self):
        ext = getattr(self, "_ext", None)
        if ext is None:
            ext = self._ext = [self.extents(j) for j in range(self.n_sys)]
        return ext

    def set_state(self, U):
        # arrays already in the ABI's layout (float64, column-major, of the
        # component's extents) are passed as they are; others are converted.
        # For hundreds of components the per-array Python work is
        # milliseconds, so the common case is kept to a few attribute checks.
        ext = self._extents_all()
        ptrs = (_lib.C.c_void_p * self.n_sys)()
        keep = []
        for j in range(self.n_sys):
            a = U[j]
            if not (type(a) is np.ndarray and a.dtype == np.float64 and a.flags.f_contiguous and a.shape == ext[j]):
                a = np.ascontiguousarray(np.asfortranarray(
                    np.broadcast_to(np.asarray(a, dtype=np.float64), ext[j])).ravel(order="F"))
                keep.append(a)
            ptrs[j] = a.ctypes.data
        check(self._L.smg_set_state(self.h, _lib.C.cast(ptrs, _lib.C.POINTER(_lib.C.POINTER(_lib.C.c_double)))),
              self.h)

    def get_state(self, which=None, out=None):
        """Components ``which`` (default all) as arrays of their extents.  With
        ``out`` ({j: float64 buffer of the component's size}, e.g. in pinned
        host memory) the values are written there."""
        return self._download(lambda ptrs: self._L.smg_get_state(self.h, ptrs), which, out)

    def snapshot(self):
        """Keep a device copy of the current state (for :meth:`get_interp`)."""
        check(self._L.smg_snapshot(self.h), self.h)

    def get_interp(self, lam, which=None, out=None):
        """Components ``which`` of ``(1 - lam) * snapshot + lam * state``,
        computed on the device (the output-time interpolation)."""
        return self._download(lambda ptrs: self._L.smg_get_interp(self.h, float(lam), ptrs), which, out)

    def _download(self, call, which, out):
        ext = self._extents_all()
        which = range(self.n_sys) if which is None else which
        res = {}
        ptrs = (_lib.C.c_void_p * self.n_sys)()
        for j in which:
            e = ext[j]
            size = e[0] * e[1] * e[2]
            if out is not None:
                buf = out[j]
                if not (type(buf) is np.ndarray and buf.dtype == np.float64 and buf.size == size
                        and (buf.flags.c_contiguous if buf.ndim == 1 else buf.flags.f_contiguous)):
                    buf = buf.reshape(-1, order="A")
                    if buf.dtype != np.float64 or buf.size != size or not buf.flags.c_contiguous:
                        raise ValueError(f"out[{j}] must be a contiguous float64 buffer of {size} values")
            else:
                buf = np.empty(size, dtype=np.float64)
            res[j] = buf
            ptrs[j] = buf.ctypes.data
        check(call(_lib.C.cast(ptrs, _lib.C.POINTER(_lib.C.POINTER(_lib.C.c_double)))), self.h)
        return {j: buf.reshape(ext[j], order="F") for j, buf in res.items()}

    def set_field(self, k, val):
        if np.ndim(val) == 0:
            check(self._L.smg_set_field(self.h, int(k), None, float(val)), self.h)
        else:
            e = self.grid_extents(self.field_grids[k])
            arr = np.ascontiguousarray(np.asfortranarray(
                np.broadcast_to(np.asarray(val, dtype=np.float64), e)).ravel(order="F"))
            check(self._L.smg_set_field(self.h, int(k), dptr(arr), 0.0), self.h)

    def set_dt(self, dt):
        check(self._L.smg_set_dt(self.h, float(dt)), self.h)

    def set_time(self, t):
        """Time of the current state (the start of the next run when sources
        are evaluated on the device)."""
        check(self._L.smg_set_time(self.h, float(t)), self.h)

    def set_material_expr(self, expr_a, expr_s0, expr_sm, rows, sA_field, EA_field, coords):
        """Evaluate the materials on the device every step
        (``smg_set_material_expr``): ``rows`` (sigma_t field, decay field,
        order m) per (grid type, order); ``coords`` six vectors, per solver
        dimension the coordinates of grid types 1 and 2.  ``expr_a=None``
        returns to uploaded values."""
        if expr_a is None:
            check(self._L.smg_set_material_expr(self.h, None, None, None, 0, None, -1, -1, None), self.h)
            return
        r = np.ascontiguousarray(np.asarray(rows, dtype=np.int32).reshape(-1))
        cs = [np.ascontiguousarray(np.asarray(c, dtype=np.float64).ravel()) for c in coords]
        ptrs = (_lib.C.POINTER(_lib.C.c_double) * 6)(*[dptr(c) for c in cs])
        check(self._L.smg_set_material_expr(self.h, expr_a.encode(), expr_s0.encode(),
                                            expr_sm.encode() if expr_sm else None, len(r) // 3, iptr(r),
                                            int(sA_field), int(EA_field), ptrs), self.h)

    def set_filter_expr(self, expr, rows, coords):
        """Evaluate the filter on the device every step (``smg_set_filter_expr``):
        ``rows`` (field at t - dt/2, field at t or -1, order k) per (grid type,
        order); ``coords`` as for :meth:`set_material_expr`.  ``expr=None``
        returns to uploaded values."""
        if expr is None:
            check(self._L.smg_set_filter_expr(self.h, None, 0, None, None), self.h)
            return
        r = np.ascontiguousarray(np.asarray(rows, dtype=np.int32).reshape(-1))
        cs = [np.ascontiguousarray(np.asarray(c, dtype=np.float64).ravel()) for c in coords]
        ptrs = (_lib.C.POINTER(_lib.C.c_double) * 6)(*[dptr(c) for c in cs])
        check(self._L.smg_set_filter_expr(self.h, expr.encode(), len(r) // 3, iptr(r), ptrs), self.h)

    def set_source_expr(self, j, expr, coords=None):
        """Evaluate the source of component j on the device every step
        (``smg_set_source_expr``): ``expr`` is a C++ expression in the solver
        coordinates x, y, z, the time t and the 1-based component k;
        ``coords`` the component's coordinate vectors per solver dimension.
        ``expr=None`` returns to uploaded source values."""
        if expr is None:
            check(self._L.smg_set_source_expr(self.h, int(j), None, None, None, None), self.h)
            return
        cs = [np.ascontiguousarray(np.asarray(c, dtype=np.float64).ravel()) for c in coords]
        e = self.extents(j)
        if any(c.size != e[d] for d, c in enumerate(cs)):
            raise ValueError(f"coordinate vectors must have the component's extents {e}")
        check(self._L.smg_set_source_expr(self.h, int(j), expr.encode(), dptr(cs[0]), dptr(cs[1]), dptr(cs[2])),
              self.h)

    def active_variant(self):
        """(kernel family the next run uses, text): with the generated kernels
        active the text names their form ("bulk-staged", "async-staged" or
        "register"), else
        the reason AUTO could not use them."""
        v = _lib.C.c_int32()
        why = _lib.C.create_string_buffer(512)
        check(self._L.smg_active_variant(self.h, _lib.C.byref(v), why, 512), self.h)
        return v.value, why.value.decode()

    def set_variant(self, variant):
        check(self._L.smg_set_variant(self.h, int(variant)), self.h)

    def tune(self, key, value):
        check(self._L.smg_tune(self.h, int(key), int(value)), self.h)

    def run(self, nsteps):
        check(self._L.smg_run(self.h, int(nsteps)), self.h)

    def sync(self):
        check(self._L.smg_sync(self.h), self.h)

    def last_run_stats(self):
        ms = _lib.C.c_double()
        nl = _lib.C.c_int64()
        check(self._L.smg_last_run_stats(self.h, _lib.C.byref(ms), _lib.C.byref(nl)), self.h)
        return ms.value, nl.value

    def layout(self):
        b = _lib.C.c_int64()
        d = (_lib.C.c_int64 * 4)()
        check(self._L.smg_layout(self.h, _lib.C.byref(b), d), self.h)
        return b.value, list(d)

    # -- discrete adjoint (smg_forward / smg_misfit / smg_backward) -----------
    def forward(self, nsteps, ckpt_every):
        check(self._L.smg_forward(self.h, int(nsteps), int(ckpt_every)), self.h)

    def misfit(self, obs):
        arr = np.ascontiguousarray(np.asfortranarray(
            np.broadcast_to(np.asarray(obs, dtype=np.float64), self.extents(0))).ravel(order="F"))
        J = _lib.C.c_double()
        check(self._L.smg_misfit(self.h, dptr(arr), _lib.C.byref(J)), self.h)
        return J.value

    def adjoint_bytes(self):
        b = _lib.C.c_int64()
        check(self._L.smg_adjoint_bytes(self.h, _lib.C.byref(b)), self.h)
        return b.value

    def adjoint_segment(self):
        """Checkpoint segment length K of the last forward."""
        k = _lib.C.c_int64()
        check(self._L.smg_adjoint_info(self.h, _lib.C.byref(k), None), self.h)
        return k.value

    def adjoint_seed(self, lam):
        arrs = []
        ptrs = (_lib.C.POINTER(_lib.C.c_double) * self.n_sys)()
        for j in range(self.n_sys):
            if lam[j] is None:
                continue
            a = np.ascontiguousarray(np.asfortranarray(
                np.broadcast_to(np.asarray(lam[j], dtype=np.float64), self.extents(j))).ravel(order="F"))
            arrs.append(a)
            ptrs[j] = dptr(a)
        check(self._L.smg_adjoint_seed(self.h, ptrs), self.h)

    def backward(self, fields=()):
        """dJ/dU(0) per component and dJ/d(field) for the requested field indices."""
        gu = {}
        pu = (_lib.C.POINTER(_lib.C.c_double) * self.n_sys)()
        for j in range(self.n_sys):
            e = self.extents(j)
            gu[j] = (np.empty(int(np.prod(e))), e)
            pu[j] = dptr(gu[j][0])
        nf = len(self.field_grids)
        pf = (_lib.C.POINTER(_lib.C.c_double) * max(nf, 1))()
        gf = {}
        scalar = getattr(self, "field_scalar", [False] * nf)
        for k in fields:
            # a scalar coefficient's derivative is one number (its sum over the points it acts on)
            gf[k] = np.empty(1 if scalar[k] else int(np.prod(self.grid_extents(self.field_grids[k]))))
            pf[k] = dptr(gf[k])
        check(self._L.smg_backward(self.h, pu, pf), self.h)
        gradU = {j: b.reshape(e, order="F") for j, (b, e) in gu.items()}
        gradF = {k: (float(v[0]) if scalar[k] else v.reshape(self.grid_extents(self.field_grids[k]), order="F"))
                 for k, v in gf.items()}
        return gradU, gradF

    def state_sumsq(self):
        out = np.zeros(self.n_sys)
        check(self._L.smg_state_sumsq(self.h, dptr(out)), self.h)
        return out

    def check_finite(self):
        return self._L.smg_check_finite(self.h)

    def close(self):
        if getattr(self, "h", None):
            if getattr(self, "owned", True):
                self._L.smg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def C_cast_fields(fa):
    return _lib.C.cast(fa, _lib.C.POINTER(_lib.smg_field))


def jit_source(n, bc, h, gt, Mx, My, Mz, fields, sigma_t, sigma_a, source, decay_t=None, decay_a=-1,
               filter_mode=FILTER_NONE, filter1=None, filter2=None, compile=False, tune=None):
    """CUDA C++ source of the problem's specialised kernels (SMG_VARIANT_JIT)
    for the SMG_TUNE_JIT_* settings in ``tune`` ({key: value}); with
    compile=True (1) also compiled by NVRTC for sm_100a (no GPU needed);
    compile=2 adds the adjoint's recording and backward-phase kernels,
    compile=3 the batched solver's family kernels."""
    L = _lib.lib()
    p, keep, _ = build_problem(n, bc, h, gt, Mx, My, Mz, fields, sigma_t, sigma_a, source,
                               decay_t, decay_a, filter_mode, filter1, filter2)
    tune = dict(tune or {})
    keys = (_lib.C.c_int32 * max(len(tune), 1))(*[int(k) for k in tune])
    vals = (_lib.C.c_int32 * max(len(tune), 1))(*[int(v) for v in tune.values()])
    ln = _lib.C.c_int64()
    check(L.smg_jit_source(_lib.C.byref(p), keys, vals, len(tune), int(compile) if int(compile) >= 2 else 0, None, 0,
                           _lib.C.byref(ln)))
    buf = _lib.C.create_string_buffer(ln.value + 1)
    check(L.smg_jit_source(_lib.C.byref(p), keys, vals, len(tune), int(compile), buf, ln.value + 1,
                           _lib.C.byref(ln)))
    return buf.value.decode()


def build_problem(n, bc, h, gt, Mx, My, Mz, fields, sigma_t, sigma_a, source,
                  decay_t=None, decay_a=-1, filter_mode=FILTER_NONE, filter1=None, filter2=None):
    """``smg_problem`` for the C ABI plus the arrays it points to (keep them
    alive until ``smg_create`` returns) and shape info for state transfers."""
    n_sys = int(np.asarray(Mz).shape[0])
    n = [int(v) for v in n]
    bc = [int(v) for v in bc]
    gt = np.ascontiguousarray(np.asarray(gt, dtype=np.int32).reshape(n_sys, 3))
    keep = []

    def i32(a):
        arr = np.ascontiguousarray(np.asarray(a, dtype=np.int32))
        keep.append(arr)
        return arr

    mats = [np.asfortranarray(np.asarray(M, dtype=np.float64)) for M in (Mx, My, Mz)]
    keep += mats
    fa = (_lib.smg_field * max(len(fields), 1))()
    keep.append(fa)
    for k, (val, grid) in enumerate(fields):
        fa[k].grid[:] = [int(g) for g in grid]
        if np.ndim(val) == 0:
            fa[k].data = None
            fa[k].scalar = float(val)
        else:
            arr = np.ascontiguousarray(np.asfortranarray(np.asarray(val, dtype=np.float64)).ravel(order="F"))
            keep.append(arr)
            fa[k].data = dptr(arr)
            fa[k].scalar = 0.0
    p = _lib.smg_problem()
    p.n_sys = n_sys
    p.n[:] = n
    p.bc[:] = bc
    p.h[:] = [float(v) for v in h]
    p.gt = iptr(i32(gt.ravel()))
    p.Mx, p.My, p.Mz = (dptr(m) for m in mats)
    p.n_fields = len(fields)
    p.fields = C_cast_fields(fa)
    p.sigma_t = iptr(i32(sigma_t))
    p.decay_t = iptr(i32(decay_t)) if decay_t is not None else None
    p.sigma_a = int(sigma_a)
    p.decay_a = int(decay_a)
    p.source = iptr(i32(source))
    p.filter_mode = int(filter_mode)
    p.filter1 = iptr(i32(filter1)) if filter1 is not None else None
    p.filter2 = iptr(i32(filter2)) if filter2 is not None else None
    info = (n_sys, n, bc, gt, [tuple(int(g) for g in grid) for _, grid in fields])
    return p, keep, info


# ----------------------------------------------------------------------
# Reference setup (starmap_solver.m:55-305) and the loop driver
# ----------------------------------------------------------------------
class _Setup:
    pass


def _as_field(v, shape):
    a = np.asarray(v, dtype=np.float64)
    if a.ndim == 0:
        return np.float64(a)
    return np.broadcast_to(a, shape)


def prepare(par: dict) -> _Setup:
    """Host-side setup of starmap_solver.m:55-157 (no GPU work)."""
    S = _Setup()
    par = dict(par)
    # the coupling matrices in the C ABI's column-major layout (MATLAB's), once
    Mx, My, Mz = (np.asfortranarray(np.asarray(par[k], dtype=np.float64)) for k in ("Mx", "My", "Mz"))
    n_sys = Mz.shape[0]
    flag_filter = ("filterfunction" in par) and ("f_position" in par) and ("mom_order" in par)
    f_mom_order = np.atleast_1d(np.asarray(par["mom_order"])).astype(int) if "mom_order" in par else None
    if not flag_filter:
        par["filterfunction"] = _ones
        par["f_position"] = ""
    flag_ani = ("sigma_sm" in par) and ("mom_order" in par)
    if not flag_ani:
        par["mom_order"] = np.concatenate([[0], np.ones(n_sys - 1, dtype=int)])
        par["sigma_sm"] = zero
    mom_order = np.atleast_1d(np.asarray(par["mom_order"])).astype(int)
    mo = par.get("mom_output", 1)
    if isinstance(mo, str) and mo == "all":
        mo = np.arange(1, n_sys + 1)
    S.mom_output = [int(v) for v in np.atleast_1d(mo)]
    gt = _lib.classify(Mx, My, Mz)
    ax = np.asarray(par["ax"], dtype=np.float64)
    n = np.asarray(par["n"], dtype=int)
    bc = np.asarray(par["bc"], dtype=int)
    h = (ax[[1, 3, 5]] - ax[[0, 2, 4]]) / n
    lam = np.max(np.abs(np.linalg.eigvals(Mz)))
    dt_hyp = np.min(h) / abs(lam)
    if n[0] != 1:
        dt_hyp = dt_hyp / 3
    elif n[1] != 1:
        dt_hyp = dt_hyp / 2
    S.timestep = int(par.get("timestep", 0))
    if S.timestep not in (0, 1, 2):
        raise ValueError("timestep must be 0 (hyperbolic), 1 or 2 (parabolic)")
    S.time_dependent = np.array([nargin(par["sigma_a"]) > 3, nargin(par["sigma_s0"]) > 3,
                                 nargin(par["sigma_sm"]) > 4])
    xs = [colon(ax[0] + h[0] / 2, h[0], ax[1] - h[0] / 2), colon(ax[0] + h[0] * (1 - bc[0]), h[0], ax[1])]
    ys = [colon(ax[2] + h[1] / 2, h[1], ax[3] - h[1] / 2), colon(ax[2] + h[1] * (1 - bc[1]), h[1], ax[3])]
    zs = [colon(ax[4] + h[2] / 2, h[2], ax[5] - h[2] / 2), colon(ax[4] + h[2] * (1 - bc[2]), h[2], ax[5])]
    grids = {}

    def XYZ(g):
        if g not in grids:
            # column-major (the reference's layout): hook results computed
            # elementwise on these grids are column-major too, so the state
            # and field uploads need no transposing copy
            grids[g] = [np.asfortranarray(a) for a in
                        np.meshgrid(xs[g[0] - 1], ys[g[1] - 1], zs[g[2] - 1], indexing="ij")]
        return grids[g]

    S.par, S.n_sys, S.Mx, S.My, S.Mz = par, n_sys, Mx, My, Mz
    S.gt, S.n, S.bc, S.h, S.dt_hyp = gt, n, bc, h, dt_hyp
    S.xs, S.ys, S.zs, S.XYZ = xs, ys, zs, XYZ
    S.mom_order, S.f_mom_order = mom_order, f_mom_order
    S.flag_filter, S.flag_ani = flag_filter, flag_ani
    S.f_position = par["f_position"]
    S.G = lambda j: (int(gt[j, 0]), int(gt[j, 1]), int(gt[j, 2]))
    S.sg = sorted(set((*S.G(j), int(mom_order[j])) for j in range(1, n_sys)))
    S.f_sg = sorted(set((*S.G(j), int(f_mom_order[j])) for j in range(1, n_sys))) if flag_filter else []
    # initial condition (starmap_solver.m:140-146)
    ic = par["ic"]
    per_moment = nargin(ic) > 3
    U, higher = [], {}
    for j in range(n_sys):
        g = S.G(j)
        X, Y, Z = XYZ(g)
        if per_moment or j == 0:
            val = capargs(ic, X, Y, Z, j + 1)
            U.append(X * 0 + np.asarray(val, dtype=np.float64) * 1.0)
            continue
        # a higher moment of an initial condition with at most three
        # arguments: X*0 + ic(X,Y,Z)*0, which the call's arguments fix per
        # grid, so it is evaluated once per grid and copied
        if g not in higher:
            higher[g] = X * 0 + np.asarray(capargs(ic, X, Y, Z, j + 1), dtype=np.float64) * 0.0
        U.append(higher[g].copy(order="K"))
    S.U0 = U
    if S.timestep > 0:
        S.M_sym = timestep.symbol(Mx, My, Mz, h)
        n2 = np.sum(gt == 2, axis=1)
        S.even = [j for j in range(n_sys) if n2[j] % 2 == 0]     # c111, c221, c212, c122
        S.odd = [j for j in range(n_sys) if n2[j] % 2 == 1]      # c211, c121, c112, c222
    S.source_ind = [int(v) for v in np.atleast_1d(np.asarray(par.get("source_ind", [])))]
    S.src_td = nargin(par["source"]) >= 4 and len(S.source_ind) > 0
    S.filter_td = flag_filter and nargin(par["filterfunction"]) > 6
    return S


def _ones(*args):
    return 1.0


_ones._nargin = -1


def _materials(S, t):
    """sA{g}, sT{g,m} evaluated at time t (starmap_solver.m:215-243)."""
    par = S.par
    grids_used = sorted(set([(1, 1, 1)] + [row[:3] for row in S.sg]))
    sA = {g: _as_field(capargs(par["sigma_a"], *S.XYZ(g), t), S.XYZ(g)[0].shape) for g in grids_used}
    sT = {}
    for row in S.sg:
        g, m = row[:3], row[3]
        X, Y, Z = S.XYZ(g)
        sS = np.asarray(capargs(par["sigma_s0"], X, Y, Z, t), dtype=np.float64)
        if S.flag_ani:
            sS = sS - np.asarray(capargs(par["sigma_sm"], X, Y, Z, m, t), dtype=np.float64)
        sT[row] = _as_field(sA[g] + sS, X.shape)
    return sA, sT


def _filters(S, dt, t):
    par = S.par
    F = {}
    for row in S.f_sg:
        g, m = row[:3], row[3]
        X, Y, Z = S.XYZ(g)
        if S.f_position == "full":
            F[row] = _as_field(capargs(par["filterfunction"], par, dt, m, X, Y, Z, t), X.shape)
        elif S.f_position == "substep":
            F[row + (1,)] = _as_field(capargs(par["filterfunction"], par, dt, m, X, Y, Z, t - dt / 2), X.shape)
            F[row + (2,)] = _as_field(capargs(par["filterfunction"], par, dt, m, X, Y, Z, t), X.shape)
    return F


def _sources(S, t, dt):
    par = S.par
    Q = {}
    for j1 in S.source_ind:
        j = j1 - 1
        X, Y, Z = S.XYZ(S.G(j))
        Q[j] = _as_field(capargs(par["source"], X, Y, Z, t - dt / 2, j1), X.shape)
    return Q


class _Tables:
    """Field table of the C ABI with stable indices for later updates."""

    def __init__(self):
        self.fields = []
        self.index = {}

    def add(self, key, val, grid):
        # arrays in the C ABI's column-major layout once, here, rather than
        # at every handle creation
        if np.ndim(val) > 0:
            val = np.asfortranarray(np.asarray(val, dtype=np.float64))
        self.index[key] = len(self.fields)
        self.fields.append((val, grid))
        return self.index[key]


def _build(S, sA1, sT1, EA, ET, Q, F):
    T = _Tables()
    for row in S.sg:
        T.add(("sT",) + row, sT1[row], row[:3])
        T.add(("ET",) + row, ET[row], row[:3])
    T.add(("sA",), sA1, (1, 1, 1))
    T.add(("EA",), EA, (1, 1, 1))
    for j, q in Q.items():
        T.add(("Q", j), q, S.G(j))
    for key, val in F.items():
        T.add(("F",) + key, val, key[:3])
    solver = GpuSolver(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, T.fields, **handle_tables(S, T))
    if DEFAULT_VARIANT != VARIANT_AUTO:
        solver.set_variant(DEFAULT_VARIANT)
    return solver, T


def handle_tables(S, T) -> dict:
    """Per-component field indices of the C-ABI descriptor for setup ``S`` and table ``T``."""
    n_sys = S.n_sys
    key = lambda j: (*S.G(j), int(S.mom_order[j]))
    sigma_t = [0] + [T.index[("sT",) + key(j)] for j in range(1, n_sys)]
    decay_t = [0] + [T.index[("ET",) + key(j)] for j in range(1, n_sys)]
    source = [T.index.get(("Q", j), -1) for j in range(n_sys)]
    mode = {"": FILTER_NONE, "substep": FILTER_SUBSTEP, "full": FILTER_FULL}.get(S.f_position, FILTER_NONE)
    if not S.flag_filter:
        mode = FILTER_NONE
    f1 = f2 = None
    if mode != FILTER_NONE:
        fkey = lambda j: (*S.G(j), int(S.f_mom_order[j]))
        if mode == FILTER_SUBSTEP:
            f1 = [-1] + [T.index[("F",) + fkey(j) + (1,)] for j in range(1, n_sys)]
            f2 = [-1] + [T.index[("F",) + fkey(j) + (2,)] for j in range(1, n_sys)]
        else:
            f1 = [-1] + [T.index[("F",) + fkey(j)] for j in range(1, n_sys)]
    return dict(sigma_t=sigma_t, sigma_a=T.index[("sA",)], source=source, decay_t=decay_t,
                decay_a=T.index[("EA",)], filter_mode=mode, filter1=f1, filter2=f2)


def _output_struct(S, U):
    dim = S.par.get("dim", 3)
    out = []
    for j in range(S.n_sys):
        g = S.G(j)
        if dim == 1:
            out.append({"x": S.zs[g[2] - 1], "U": U[j].reshape(len(S.zs[g[2] - 1]), -1, order="F")})
        elif dim == 2:
            out.append({"x": S.ys[g[1] - 1], "y": S.zs[g[2] - 1],
                        "U": U[j].reshape(len(S.ys[g[1] - 1]), -1, order="F")})
        else:
            out.append({"x": S.xs[g[0] - 1], "y": S.ys[g[1] - 1], "z": S.zs[g[2] - 1], "U": U[j]})
    return out


def step_materials(S, t, dt_prev, sA, sT):
    """dt and the materials of the step from time t (starmap_solver.m:168-265):
    the hyperbolic step, or with ``timestep > 0`` the parabolic search from
    the materials at t; for time-dependent materials those at t + dt,
    averaged with the ones at t (with the parabolic step, falling back to the
    ones at t when the average is unstable).  Returns
    ``(dt, sA, sT, sA1, sT1)`` with sA, sT the materials to carry to the next step."""
    tfinal = float(S.par["tfinal"])
    cn = float(S.par["cn"])
    tleft = (tfinal - t) / cn
    la0 = None
    if S.timestep > 0:
        decay = timestep.decay_vector(S.n_sys, S.gt, S.mom_order, sA[1, 1, 1], sT)
        dt_b, la0 = timestep.search(S.M_sym, S.even, S.odd, decay, dt_prev, S.dt_hyp, tleft, S.timestep)
    else:
        dt_b = S.dt_hyp
    dt = min(dt_b, tleft) * cn
    if not S.time_dependent.any():
        return dt, sA, sT, sA[1, 1, 1], sT
    sA0, sT0 = sA, sT
    sA, sT = _materials(S, t + dt)
    sA1 = (sA0[1, 1, 1] + sA[1, 1, 1]) / 2
    sT1 = {k: (sT0[k] + sT[k]) / 2 for k in S.sg}
    if S.timestep > 0:
        decay = timestep.decay_vector(S.n_sys, S.gt, S.mom_order, sA1, sT1)
        if not timestep.stable(S.M_sym, S.even, S.odd, decay, dt, la0, S.timestep):
            sA1, sT1 = sA0[1, 1, 1], sT0
    return dt, sA, sT, sA1, sT1


def first_step(S):
    """Materials, dt, decay factors, source and filter tables as the reference
    evaluates them for the first step (starmap_solver.m:165-305)."""
    sA, sT = _materials(S, 0.0)
    dt, sA, sT, sA1, sT1 = step_materials(S, 0.0, 0.0, sA, sT)
    EA = expm1div(-sA1 * dt / 2)
    ET = {k: expm1div(-sT1[k] * dt / 2) for k in S.sg}
    Q = _sources(S, dt, dt)
    F = _filters(S, dt, dt) if S.flag_filter else {}
    return dict(sA=sA, sT=sT, sA1=sA1, sT1=sT1, EA=EA, ET=ET, dt=dt, Q=Q, F=F)


def setup_gpu(par: dict):
    """Host setup plus library handle for ``par`` (state and dt not yet set).

    Returns ``(S, fs, solver, table)``: the setup, the first-step data, the
    :class:`GpuSolver` and the field table (for later ``set_field`` calls)."""
    S = prepare(par)
    fs = first_step(S)
    solver, T = _build(S, fs["sA1"], fs["sT1"], fs["EA"], fs["ET"], fs["Q"], fs["F"])
    return S, fs, solver, T


def starmap_solver(par: dict):
    """Run the StaRMAP time loop on the GPU; returns the reference's ``output``.

    ``output[j]`` is a dict with keys ``x``, ``y`` (2D), ``z`` (3D) and ``U`` for
    component j+1, exactly the struct array of starmap_solver.m:484-500."""
    t_start = time.perf_counter()
    S = prepare(par)
    par = S.par
    tfinal = float(par["tfinal"])
    cn = float(par["cn"])
    td_any = bool(S.time_dependent.any())
    fs = first_step(S)
    sA, sT, sA1, sT1, dt = fs["sA"], fs["sT"], fs["sA1"], fs["sT1"], fs["dt"]
    cpu_setup = time.perf_counter() - t_start

    # a time-dependent source given also as an expression is evaluated on the
    # device every step instead of on the host; so are time-dependent
    # materials when every material hook has an expression (hyperbolic dt,
    # filters not time-dependent)
    dev_src = bool(S.src_td) and bool(par.get("source_expr"))
    dev_filt = bool(S.filter_td) and bool(par.get("filterfunction_expr"))
    dev_mat = (td_any and S.timestep == 0 and (dev_filt or not S.filter_td) and (dev_src or not S.src_td)
               and bool(par.get("sigma_a_expr")) and bool(par.get("sigma_s0_expr"))
               and (bool(par.get("sigma_sm_expr")) or not S.flag_ani))
    # fields written by the device every step become arrays
    shape = lambda g: S.XYZ(g)[0].shape
    full = lambda v, g: np.ascontiguousarray(np.broadcast_to(np.asarray(v, dtype=np.float64), shape(g)))
    Fv = {k: full(v, k[:3]) for k, v in fs["F"].items()} if dev_filt else fs["F"]
    if dev_mat:
        solver, T = _build(S, full(sA1, (1, 1, 1)), {k: full(v, k[:3]) for k, v in sT1.items()},
                           full(fs["EA"], (1, 1, 1)), {k: full(v, k[:3]) for k, v in fs["ET"].items()},
                           fs["Q"], Fv)
    else:
        solver, T = _build(S, sA1, sT1, fs["EA"], fs["ET"], fs["Q"], Fv)
    t_gpu0 = time.perf_counter()
    try:
        solver.set_state(S.U0)
        solver.set_dt(dt)
        if dev_src:
            expr = device_source_expr(par["source_expr"], int(par.get("dim", 3)))
            for j1 in S.source_ind:
                g = S.G(j1 - 1)
                solver.set_source_expr(j1 - 1, expr, [S.xs[g[0] - 1], S.ys[g[1] - 1], S.zs[g[2] - 1]])
            solver.set_time(0.0)
        coords6 = [S.xs[0], S.xs[1], S.ys[0], S.ys[1], S.zs[0], S.zs[1]]
        if dev_filt:
            if S.f_position == "substep":
                frows = [(T.index[("F",) + row + (1,)], T.index[("F",) + row + (2,)], row[3]) for row in S.f_sg]
            else:
                frows = [(T.index[("F",) + row], -1, row[3]) for row in S.f_sg]
            solver.set_filter_expr(device_source_expr(par["filterfunction_expr"], int(par.get("dim", 3))),
                                   frows, coords6)
            solver.set_time(0.0)
        if dev_mat:
            dim = int(par.get("dim", 3))
            ex = lambda key: device_source_expr(par[key], dim) if par.get(key) else None
            rows = [(T.index[("sT",) + row], T.index[("ET",) + row], row[3]) for row in S.sg]
            solver.set_material_expr(ex("sigma_a_expr"), ex("sigma_s0_expr"),
                                     ex("sigma_sm_expr") if S.flag_ani else None, rows, T.index[("sA",)],
                                     T.index[("EA",)], [S.xs[0], S.xs[1], S.ys[0], S.ys[1], S.zs[0], S.zs[1]])
            solver.set_time(0.0)
            sched_t, sched_dt = td_schedule(S.dt_hyp, tfinal, cn)
        t_plot = list(np.atleast_1d(np.asarray(par.get("t_plot", [])))) + [np.inf]
        want_plot = par.get("output", _noop_output) is not _noop_output
        per_step = (td_any and not dev_mat) or (S.src_td and not dev_src) or (S.filter_td and not dev_filt)
        step_count = 0
        t_cur = 0.0
        plot_count = 0
        outfn = par.get("output", _noop_output)
        while t_cur < tfinal:
            if per_step and step_count > 0:
                # time-dependent data re-evaluated where the reference does
                if td_any:
                    dt_new, sA, sT, sA1, sT1 = step_materials(S, t_cur, dt, sA, sT)
                    if dt_new != dt:
                        dt = dt_new
                        solver.set_dt(dt)
                    solver.set_field(T.index[("sA",)], sA1)
                    solver.set_field(T.index[("EA",)], expm1div(-sA1 * dt / 2))
                    for k in S.sg:
                        solver.set_field(T.index[("sT",) + k], sT1[k])
                        solver.set_field(T.index[("ET",) + k], expm1div(-sT1[k] * dt / 2))
                tn = t_cur + dt
                if S.src_td and not dev_src:
                    for j, q in _sources(S, tn, dt).items():
                        solver.set_field(T.index[("Q", j)], q)
                if S.filter_td and not dev_filt:
                    for key, val in _filters(S, dt, tn).items():
                        solver.set_field(T.index[("F",) + key], val)
            # how many steps can run before the next plot time
            if per_step:
                nrun = 1
            elif dev_mat:
                ts, dts = sched_t[step_count:], sched_dt[step_count:]
                if dts[0] != dt:
                    dt = dts[0]
                    solver.set_dt(dt)
                nrun = 1
                while nrun < len(dts) and dts[nrun] == dts[0]:
                    nrun += 1
                ts = ts[:nrun]
            else:
                ts = step_times(dt, tfinal)[step_count:]
                nrun = len(ts)
            if not per_step and want_plot:
                for k, tk in enumerate(ts):
                    if tk >= t_plot[plot_count] - 1e-14:
                        nrun = k + 1
                        break
            if want_plot and nrun >= 1:
                if nrun > 1:
                    solver.run(nrun - 1)
                    for _ in range(nrun - 1):
                        t_cur = t_cur + dt
                    step_count += nrun - 1
                    nrun = 1
                solver.snapshot()   # the state before the last step, kept on the device
            solver.run(nrun)
            for _ in range(nrun):
                t_cur = t_cur + dt
            step_count += nrun
            if want_plot:
                while t_cur >= t_plot[plot_count] - 1e-14:
                    lam = (t_plot[plot_count] - t_cur + dt) / dt
                    # (1 - lam) * U0 + lam * Un on the device, downloaded once
                    Ud = solver.get_interp(lam, [j - 1 for j in S.mom_output])
                    Uplot = [Ud[j - 1] for j in S.mom_output]
                    ret = _call_output(S, outfn, par, Uplot, plot_count + 1)
                    if isinstance(ret, dict):
                        par = ret
                        S.par = par
                    plot_count += 1
        Ufin = solver.get_state()
    finally:
        solver.close()
    gpu_s = time.perf_counter() - t_gpu0
    U = [Ufin[j] for j in range(S.n_sys)]
    if not par.get("quiet", False):
        n = list(S.n)
        print(f"{par.get('name', 'Output')} with {par.get('closure_mod', '')}{par['closure']}{par['n_mom']}\n"
              f" {S.n_sys} moments, {n[0]}x{n[1]}x{n[2]} grid, {step_count} time steps")
        tot = max(cpu_setup + gpu_s, 1e-30)
        print(f"CPU-times\n advection:{gpu_s:12.2f}s{gpu_s / tot * 100:5.0f}%\n "
              f"absorb/scatter:{cpu_setup:7.2f}s{cpu_setup / tot * 100:5.0f}%\n plotting:{0.0:13.2f}s{0:5.0f}%")
    return _output_struct(S, U)


def td_schedule(dt_hyp: float, tfinal: float, cn: float):
    """Times after each step and the dt of each step as the reference chooses
    them for time-dependent materials with the hyperbolic step
    (starmap_solver.m:165-209): dt = min(dt_hyp, time left / cn) * cn, so the
    last step is shortened to end at tfinal, and t = t + dt."""
    ts, dts = [], []
    t = 0.0
    while t < tfinal:
        d = min(dt_hyp, (tfinal - t) / cn) * cn
        t = t + d
        ts.append(t)
        dts.append(d)
    return ts, dts


_IDENT = re.compile(r"(?<![\w.])[A-Za-z_]\w*")


def device_source_expr(expr: str, dim: int) -> str:
    """The user's device expression, written in the variables of the user's
    own hook (x, y, t, k in 2D; x, y, z, t, k in 3D; x, t, k in 1D), as an
    expression in the solver dimensions that ``smg_set_source_expr`` and the
    other device-expression calls take: in 2D the user's (x, y) are the
    solver's second and third dimensions, in 1D the user's x is the third
    (the wrapping of starmap_init.m).  The variables are renamed token by
    token (identifiers inside numbers such as 1e5 or 0x1p-3 are not
    tokens); a variable the user's hook does not have is refused."""
    if dim == 3:
        return "(" + expr + ")"
    ren = {"x": "y", "y": "z"} if dim == 2 else {"x": "z"}
    absent = {"z"} if dim == 2 else {"y", "z"}

    def sub(m):
        w = m.group(0)
        if w in absent:
            raise ValueError(f"device expression {expr!r}: '{w}' is not a variable of a {dim}D problem")
        return ren.get(w, w)

    return "(" + _IDENT.sub(sub, expr) + ")"


def _call_output(S, outfn, par, Uplot, step):
    """Plot callback with the reference's argument layout (starmap_solver.m:432-471)."""
    dim = par.get("dim", 3)
    mo = [j - 1 for j in S.mom_output]
    if dim == 1:
        zp = [S.zs[S.gt[j, 2] - 1] for j in mo]
        Up = [u.reshape(len(z), -1, order="F") for u, z in zip(Uplot, zp)]
        if len(mo) == 1:
            zp, Up = zp[0], Up[0]
        return outfn(par, zp, Up, step)
    if dim == 2:
        yp = [S.ys[S.gt[j, 1] - 1] for j in mo]
        zp = [S.zs[S.gt[j, 2] - 1] for j in mo]
        Up = [u.reshape(len(y), -1, order="F") for u, y in zip(Uplot, yp)]
        if len(mo) == 1:
            yp, zp, Up = yp[0], zp[0], Up[0]
        return outfn(par, yp, zp, Up, step)
    xp = [S.xs[S.gt[j, 0] - 1] for j in mo]
    yp = [S.ys[S.gt[j, 1] - 1] for j in mo]
    zp = [S.zs[S.gt[j, 2] - 1] for j in mo]
    Up = list(Uplot)
    if len(mo) == 1:
        xp, yp, zp, Up = xp[0], yp[0], zp[0], Up[0]
    return outfn(par, xp, yp, zp, Up, step)

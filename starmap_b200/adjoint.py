"""Gradients of an L2 misfit on the zeroth moment through the GPU time loop.

``MisfitAdjoint`` is a forward/backward pair in the shape of an autograd
function, without a tensor framework (the reference's host is MATLAB/Octave):

    adj = MisfitAdjoint(par)             # ckpt_every=0: record as much as memory allows
    J = adj.forward(obs, nsteps)      # J = 1/2 sum (U_1(T) - obs)^2
    g = adj.backward()                # dict of gradients
    adj.close()

``g["sigma_a"][grid]`` and ``g["sigma_s0"][grid]`` are the derivatives with
respect to the coefficient samples on each staggered grid ``grid`` (the
reference samples sigma_a and sigma_s0 separately on every grid type,
starmap_solver.m:215-243; a user field defined on the domain gets its gradient
by summing these through its own sampling), ``g["source"][j]`` for every
component with a source, ``g["ic"][j]`` for every component, ``g["J"]`` the
misfit.  Scalar coefficients get scalar derivatives.

``ckpt_every=K`` keeps a checkpoint every K steps and recomputes each segment
during the backward sweep (memory: about K recorded steps); ``ckpt_every=0``
picks the largest K that fits in device memory, normally the whole run, so
that nothing is recomputed.  ``last_ms()`` is the device time of the last
forward or backward call.
"""
from __future__ import annotations

import numpy as np

from .batch import _tables
from .solver import GpuSolver, first_step, handle_tables, prepare

__all__ = ["MisfitAdjoint", "batched_gradients"]


class MisfitAdjoint:
    def __init__(self, par: dict, ckpt_every: int = 0):
        S = prepare(par)
        if S.time_dependent.any() or S.src_td or S.filter_td:
            raise NotImplementedError("the adjoint covers autonomous problems")
        self.S = S
        self.fs = first_step(S)
        self.T = _tables(S, self.fs)
        self.solver = GpuSolver(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, self.T.fields,
                                **handle_tables(S, self.T))
        self.ckpt_every = int(ckpt_every)
        self.J = None

    def forward(self, obs, nsteps: int, U0=None) -> float:
        s = self.solver
        s.set_state(self.S.U0 if U0 is None else U0)
        s.set_dt(self.fs["dt"])
        s.forward(int(nsteps), self.ckpt_every)
        self.J = s.misfit(obs)
        return self.J

    def backward(self) -> dict:
        S, T = self.S, self.T
        keys = [k for k in T.index if k[0] in ("sT", "sA", "Q")]
        gU, gF = self.solver.backward(fields=[T.index[k] for k in keys])
        sig_a, sig_s0 = {}, {}

        def add(d, g, v):
            d[g] = d[g] + v if g in d else np.array(v, dtype=np.float64)

        for key in keys:
            v = gF[T.index[key]]
            if key[0] == "sT":   # sT{g,m} = sA{g} + sS0{g} - sSm{g,m}
                g = key[1:4]
                add(sig_a, g, v)
                add(sig_s0, g, v)
            elif key[0] == "sA":  # sA1 = sA{1,1,1} drives the zeroth moment
                add(sig_a, (1, 1, 1), v)
        src = {key[1]: gF[T.index[key]] for key in keys if key[0] == "Q"}
        return {"J": self.J, "sigma_a": sig_a, "sigma_s0": sig_s0, "source": src,
                "ic": [gU[j] for j in range(S.n_sys)]}

    def last_ms(self) -> float:
        return self.solver.last_run_stats()[0]

    def close(self):
        self.solver.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def batched_gradients(pars, obs, nsteps: int, ckpt_every: int = 20, threads: int = 8):
    """Misfit gradients of many independent problems (e.g. an ensemble of
    inverse problems) in one call: one :class:`MisfitAdjoint` per problem,
    their forward and backward sweeps issued from ``threads`` host threads so
    that the instances' kernels (each handle has its own CUDA stream) overlap
    on the GPU.  ``obs[i]`` is problem i's observation.  Returns the list of
    gradient dicts and the wall seconds of the forward and backward stages.
    ``ckpt_every`` must be > 0: with 0 every instance would size its
    recording to the whole free memory."""
    import time
    from concurrent.futures import ThreadPoolExecutor
    if ckpt_every < 1:
        raise ValueError("batched gradients need an explicit checkpoint interval (ckpt_every >= 1)")
    adjs = [MisfitAdjoint(p, ckpt_every=ckpt_every) for p in pars]
    try:
        with ThreadPoolExecutor(max_workers=max(1, int(threads))) as ex:
            t0 = time.perf_counter()
            list(ex.map(lambda ao: ao[0].forward(ao[1], nsteps), zip(adjs, obs)))
            t1 = time.perf_counter()
            grads = list(ex.map(lambda a: a.backward(), adjs))
            t2 = time.perf_counter()
        return grads, t1 - t0, t2 - t1
    finally:
        for a in adjs:
            a.close()

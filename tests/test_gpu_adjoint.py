"""Discrete adjoint: dot-product test (linear part), central finite
differences for the sigma, source and initial-condition gradients, the
checkpoint length not changing the result, and the fused and the two-kernel
backward sweeps agreeing."""
import numpy as np
import pytest

from starmap_b200 import _lib, configs, starmap_init
from starmap_b200.batch import _tables
from starmap_b200.solver import GpuSolver, expm1div, first_step, handle_tables, prepare

pytestmark = pytest.mark.gpu


def adjoint_problem(n=12, N=3, bc=1, with_source=True, substep=True, scalar=False):
    par = adjoint_par(n, N, bc, with_source, substep, scalar)
    S = prepare(par)
    fs = first_step(S)
    return S, fs


def adjoint_par(n=12, N=3, bc=1, with_source=True, substep=True, scalar=False):
    def sig_a(x, y):
        return 0.4 if scalar else 0.3 + 0.2 * np.sin(2 * x) * np.cos(y)

    def sig_s(x, y):
        return 0.9 if scalar else 0.8 + 0.1 * x

    prob = dict(name="adj", closure="P", n_mom=N, ax=[-1.0, 1.0, -1.0, 1.0], n=[n, n + 2], bc=[bc, bc],
                ic=lambda x, y: np.exp(-8 * (x ** 2 + (y - 0.1) ** 2)), sigma_a=sig_a,
                sigma_s0=sig_s, tfinal=1e9, t_plot=[0, 1e9], quiet=True)
    if with_source:
        prob["source"] = lambda x, y: np.exp(-6 * ((x - 0.3) ** 2 + y ** 2))
    if substep:
        prob.update(filterfunction=configs.exp_filter(2, 3.0), f_position="substep")
    return starmap_init(prob)


def make_solver(S, fs, T=None, fused=1, variant=0):
    """variant 0 (AUTO): generated recording and backward kernels; 4: the
    precompiled pair kernel and the precompiled backward kernels."""
    T = T or _tables(S, fs)
    solver = GpuSolver(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, T.fields, **handle_tables(S, T))
    solver.tune(_lib.SMG_TUNE_ADJ_FUSED, fused)
    if variant:
        solver.set_variant(variant)
    return solver, T


def run_J(S, fs, T, U0, nsteps, obs):
    solver, _ = make_solver(S, fs, T)
    try:
        solver.set_state(U0)
        solver.set_dt(fs["dt"])
        solver.run(nsteps)
        u = solver.get_state([0])[0]
    finally:
        solver.close()
    return 0.5 * np.sum((u - obs) ** 2)


def with_sigma(T, S, fs, key, arr):
    """Field table with sigma field `key` replaced by arr and its decay recomputed."""
    import copy
    T2 = copy.copy(T)
    T2.fields = list(T.fields)
    k = T.index[key]
    T2.fields[k] = (arr, T.fields[k][1])
    dkey = ("EA",) if key == ("sA",) else ("ET",) + key[1:]
    kd = T.index[dkey]
    T2.fields[kd] = (expm1div(-arr * fs["dt"] / 2), T.fields[kd][1])
    return T2


@pytest.mark.parametrize("fused,K", [(1, 4), (0, 4), (1, 9)])
def test_dot_product(fused, K):
    S, fs = adjoint_problem(with_source=False)
    rng = np.random.default_rng(0)
    nsteps = 9
    solver, T = make_solver(S, fs, fused=fused)
    try:
        delta = [rng.standard_normal(solver.extents(j)) for j in range(S.n_sys)]
        mu = [rng.standard_normal(solver.extents(j)) for j in range(S.n_sys)]
        solver.set_state(delta)
        solver.set_dt(fs["dt"])
        solver.forward(nsteps, K)
        Ad = solver.get_state()
        solver.adjoint_seed(mu)
        lam0, _ = solver.backward()
    finally:
        solver.close()
    lhs = sum(np.sum(Ad[j] * mu[j]) for j in range(S.n_sys))
    rhs = sum(np.sum(delta[j] * lam0[j]) for j in range(S.n_sys))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs))


@pytest.mark.parametrize("bc,substep,fused", [(1, True, 1), (0, False, 1), (1, True, 0)])
def test_sigma_source_ic_gradients_vs_central_differences(bc, substep, fused):
    S, fs = adjoint_problem(bc=bc, substep=substep)
    nsteps = 8
    solver, T = make_solver(S, fs, fused=fused)
    obs = None
    try:
        solver.set_state(S.U0)
        solver.set_dt(fs["dt"])
        solver.forward(nsteps, 3)
        u = solver.get_state([0])[0]
        obs = 0.5 * u + 0.01
        J0 = solver.misfit(obs)
        keys = [k for k in T.index if k[0] in ("sT", "sA", "Q")]
        gU, gF = solver.backward(fields=[T.index[k] for k in keys])
    finally:
        solver.close()
    assert np.isclose(J0, run_J(S, fs, T, S.U0, nsteps, obs), rtol=1e-14)
    rng = np.random.default_rng(1)
    for key in keys:
        k = T.index[key]
        base = np.asarray(T.fields[k][0], dtype=np.float64)
        d = rng.standard_normal(base.shape)
        eps = 1e-6 * max(1.0, float(np.abs(base).max()))
        if key[0] == "Q":
            import copy
            Tp, Tm = copy.copy(T), copy.copy(T)
            Tp.fields, Tm.fields = list(T.fields), list(T.fields)
            Tp.fields[k] = (base + eps * d, T.fields[k][1])
            Tm.fields[k] = (base - eps * d, T.fields[k][1])
        else:
            Tp = with_sigma(T, S, fs, key, base + eps * d)
            Tm = with_sigma(T, S, fs, key, base - eps * d)
        fd = (run_J(S, fs, Tp, S.U0, nsteps, obs) - run_J(S, fs, Tm, S.U0, nsteps, obs)) / (2 * eps)
        ad = float(np.sum(gF[k] * d))
        assert abs(fd - ad) <= 1e-6 * max(abs(fd), 1e-3 * abs(J0)), (key, fd, ad)
    # initial condition, all components
    d = [rng.standard_normal(np.shape(S.U0[j])) for j in range(S.n_sys)]
    eps = 1e-6
    Up = [S.U0[j] + eps * d[j] for j in range(S.n_sys)]
    Um = [S.U0[j] - eps * d[j] for j in range(S.n_sys)]
    fd = (run_J(S, fs, T, Up, nsteps, obs) - run_J(S, fs, T, Um, nsteps, obs)) / (2 * eps)
    ad = sum(float(np.sum(gU[j] * d[j].reshape(gU[j].shape))) for j in range(S.n_sys))
    assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)


def test_checkpoint_interval_does_not_change_gradient():
    S, fs = adjoint_problem(n=10, N=5)
    res = []
    for K in (1, 4, 11, 0):
        solver, T = make_solver(S, fs)
        try:
            solver.set_state(S.U0)
            solver.set_dt(fs["dt"])
            solver.forward(11, K)
            u = solver.get_state([0])[0]
            solver.misfit(0.9 * u)
            gU, gF = solver.backward(fields=[T.index[("sA",)]])
            res.append((gU, gF))
        finally:
            solver.close()
    for gU, gF in res[1:]:
        for j in gU:
            np.testing.assert_allclose(gU[j], res[0][0][j], rtol=0, atol=1e-12 * np.abs(res[0][0][j]).max())


@pytest.mark.parametrize("bc,substep", [(1, True), (0, True), (1, False)])
def test_fused_and_split_sweeps_agree(bc, substep):
    S, fs = adjoint_problem(n=11, N=4, bc=bc, substep=substep)
    out = {}
    for fused in (0, 1):
        solver, T = make_solver(S, fs, fused=fused)
        try:
            solver.set_state(S.U0)
            solver.set_dt(fs["dt"])
            solver.forward(10, 3)
            u = solver.get_state([0])[0]
            solver.misfit(0.7 * u - 0.01)
            keys = [k for k in T.index if k[0] in ("sT", "sA", "Q")]
            out[fused] = solver.backward(fields=[T.index[k] for k in keys])
        finally:
            solver.close()
    (gU0, gF0), (gU1, gF1) = out[0], out[1]
    for j in gU0:
        np.testing.assert_allclose(gU1[j], gU0[j], rtol=0, atol=1e-12 * max(np.abs(gU0[j]).max(), 1e-300))
    for k in gF0:
        a, b = np.asarray(gF0[k]), np.asarray(gF1[k])
        np.testing.assert_allclose(b, a, rtol=0, atol=1e-12 * max(np.abs(a).max(), 1e-300))


def test_backward_reports_device_time_and_repeats():
    """smg_last_run_stats after forward/backward gives their device time; a
    second misfit+backward on the same forward gives the same gradient."""
    S, fs = adjoint_problem(n=10, N=3)
    solver, T = make_solver(S, fs)
    try:
        solver.set_state(S.U0)
        solver.set_dt(fs["dt"])
        solver.forward(6, 0)
        ms_f, nl_f = solver.last_run_stats()
        u = solver.get_state([0])[0]
        solver.misfit(0.5 * u)
        g1, _ = solver.backward()
        ms_b, nl_b = solver.last_run_stats()
        solver.misfit(0.5 * u)
        g2, _ = solver.backward()
    finally:
        solver.close()
    assert ms_f > 0 and ms_b > 0 and nl_f == 13 and nl_b > 0
    for j in g1:
        np.testing.assert_array_equal(g1[j], g2[j])


@pytest.mark.parametrize("bc,substep,fused,K,scalar,variant", [
    (1, True, 1, 3, False, 0), (0, False, 1, 0, False, 0), (1, True, 0, 4, False, 0), (1, True, 1, 2, True, 0),
    (1, True, 1, 3, False, 4), (0, True, 1, 7, True, 4)])
def test_gradients_match_cpu_adjoint(bc, substep, fused, K, scalar, variant):
    """GPU dJ/dU(0), dJ/dsigma_t, dJ/dsigma_a and dJ/dq against the oracle's
    CPU adjoint of the same loop (oracle/adjoint_np.py), relative 1e-11 per
    output array."""
    from oracle import adjoint_np as A
    S, fs = adjoint_problem(bc=bc, substep=substep, scalar=scalar)
    nsteps = 7
    solver, T = make_solver(S, fs, fused=fused, variant=variant)
    try:
        solver.set_state(S.U0)
        solver.set_dt(fs["dt"])
        solver.forward(nsteps, K)
        u = solver.get_state([0])[0]
        obs = 0.5 * u + 0.01
        J = solver.misfit(obs)
        keys = [k for k in T.index if k[0] in ("sT", "sA", "Q")]
        gU, gF = solver.backward(fields=[T.index[k] for k in keys])
    finally:
        solver.close()
    # the oracle takes the reference's par (prepare() keeps its own adjusted copy)
    ref = A.adjoint(adjoint_par(bc=bc, substep=substep, scalar=scalar), nsteps, A.misfit_seed(obs))
    assert np.isclose(J, ref["J"], rtol=1e-13)

    def close(got, want, what):
        got = np.asarray(got, dtype=np.float64).ravel(order="F")
        want = np.asarray(want, dtype=np.float64).ravel(order="F")
        err = np.linalg.norm(got - want) / max(np.linalg.norm(want), 1e-300)
        assert err <= 1e-11, (what, err)

    for j in range(S.n_sys):
        close(gU[j], ref["lam0"][j], ("U0", j))
    for key in keys:
        k = T.index[key]
        if key[0] == "sT":
            close(gF[k], ref["g_sT"][key[1:]], key)
        elif key[0] == "sA":
            close(gF[k], ref["g_sA"], key)
        else:
            close(gF[k], ref["g_Q"][key[1]], key)


def test_batched_gradients_match_one_at_a_time():
    """Many independent inverse problems through batched_gradients (host
    threads, one stream per instance, overlapping on the GPU): every
    instance's gradient equals its own MisfitAdjoint run."""
    from starmap_b200.adjoint import MisfitAdjoint, batched_gradients
    pars = [adjoint_par(n=10 + i, N=3, bc=i % 2) for i in range(5)]
    obs = [0.01 * (i + 1) for i in range(5)]
    grads, tf, tb = batched_gradients(pars, obs, nsteps=9, ckpt_every=4, threads=3)
    assert tf > 0 and tb > 0
    for par, o, g in zip(pars, obs, grads):
        a = MisfitAdjoint(par, ckpt_every=4)
        try:
            J = a.forward(o, 9)
            ref = a.backward()
        finally:
            a.close()
        assert g["J"] == J
        for j, v in enumerate(ref["ic"]):
            np.testing.assert_array_equal(g["ic"][j], v)
        for key in ("sigma_a", "sigma_s0"):
            for grid, v in ref[key].items():
                np.testing.assert_array_equal(g[key][grid], v)


@pytest.mark.parametrize("prio", [1, 2])
def test_stream_priorities_do_not_change_gradient(prio):
    """SMG_TUNE_ADJ_PRIORITY (recompute stream above the sweep, or the sweep on
    a stream of the highest priority) reorders only the overlap of recompute
    and sweep: gradients equal the default's to 1e-12 (atomics may sum in
    another order)."""
    S, fs = adjoint_problem(n=10, N=5)
    res = []
    for p in (0, prio):
        solver, T = make_solver(S, fs)
        try:
            solver.tune(_lib.SMG_TUNE_ADJ_PRIORITY, p)
            solver.set_state(S.U0)
            solver.set_dt(fs["dt"])
            solver.forward(11, 3)
            u = solver.get_state([0])[0]
            solver.misfit(0.9 * u)
            res.append(solver.backward(fields=[T.index[("sA",)]]))
        finally:
            solver.close()
    (gU0, gF0), (gU1, gF1) = res
    for j in gU0:
        np.testing.assert_allclose(gU1[j], gU0[j], rtol=0, atol=1e-12 * max(np.abs(gU0[j]).max(), 1e-300))
    for k in gF0:
        a, b = np.asarray(gF0[k]), np.asarray(gF1[k])
        np.testing.assert_allclose(b, a, rtol=0, atol=1e-12 * max(np.abs(a).max(), 1e-300))

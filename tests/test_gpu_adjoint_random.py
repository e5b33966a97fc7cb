"""Randomised GPU adjoint: hypothesis-drawn 2D/3D problems (P_N and SP_N,
orders, odd sizes, per-axis boundary conditions, fields, a source, filter
'' or 'substep') -- the GPU's dJ/dU(0), dJ/dsigma_t, dJ/dsigma_a and dJ/dq
against the CPU adjoint of the same loop, relative 1e-11 per array."""
import numpy as np
import pytest
from hypothesis import HealthCheck, assume, given, settings

from oracle import adjoint_np as A
from starmap_b200 import starmap_init
from starmap_b200.solver import first_step, prepare
from test_cpu_oracle_random import problems
from test_gpu_adjoint import make_solver

pytestmark = pytest.mark.gpu


@settings(max_examples=8, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(problems())
def test_gpu_adjoint_matches_cpu_adjoint_on_random_problems(prob):
    assume(prob.get("f_position", "") != "full")
    prob = dict(prob, tfinal=1e9)
    par = starmap_init(prob)
    S = prepare(par)
    fs = first_step(S)
    nsteps = 4
    solver, T = make_solver(S, fs)
    try:
        solver.set_state(S.U0)
        solver.set_dt(fs["dt"])
        solver.forward(nsteps, 2)
        u = solver.get_state([0])[0]
        obs = 0.5 * u + 0.01
        J = solver.misfit(obs)
        keys = [k for k in T.index if k[0] in ("sT", "sA", "Q")]
        gU, gF = solver.backward(fields=[T.index[k] for k in keys])
    finally:
        solver.close()
    ref = A.adjoint(starmap_init(prob), nsteps, A.misfit_seed(obs))
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
        elif key[1] in ref["g_Q"]:
            close(gF[k], ref["g_Q"][key[1]], key)

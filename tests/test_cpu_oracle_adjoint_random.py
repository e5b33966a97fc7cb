"""Randomised dot-product test of the CPU adjoint (the checker of the GPU
adjoint): for hypothesis-drawn 2D/3D problems (P_N and SP_N, orders, odd
sizes, per-axis boundary conditions, fields, a source, filter '' or
'substep'), <U(d) - U(0), mu> equals <d, lambda_0(mu)> -- the state map is
affine in the initial condition and the adjoint is its transpose."""
import numpy as np
from hypothesis import HealthCheck, assume, given, settings

from oracle import adjoint_np as A
from oracle import solver_np as O
from starmap_b200 import starmap_init
from test_cpu_oracle_random import problems


def _final(par, nsteps, U0):
    rec = A._Recorder(U0)
    return O.starmap_solver(par, max_steps=nsteps, advance=rec).U


@settings(max_examples=10, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(problems())
def test_oracle_adjoint_dot_product_on_random_problems(prob):
    assume(prob.get("f_position", "") != "full")
    prob = dict(prob, tfinal=1e9)
    par = starmap_init(prob)
    nsteps = 3
    shapes = [np.shape(u) for u in _final(par, 1, None)]
    rng = np.random.default_rng(11)
    delta = [rng.standard_normal(s) for s in shapes]
    mu = [rng.standard_normal(s) for s in shapes]
    out = A.adjoint(par, nsteps, lambda U: (mu, 0.0), U0=delta)
    c = _final(par, nsteps, [np.zeros(s) for s in shapes])
    lhs = sum(float(np.sum((u - c0) * m)) for u, c0, m in zip(out["U"], c, mu))
    rhs = sum(float(np.sum(d * l)) for d, l in zip(delta, out["lam0"]))
    assert abs(lhs - rhs) <= 1e-11 * max(abs(lhs), abs(rhs), 1e-300)

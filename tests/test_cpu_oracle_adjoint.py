"""The CPU adjoint of the oracle (oracle/adjoint_np.py) checked on its own:
dot-product test against the oracle's forward loop, and central finite
differences of the oracle's misfit for the sigma, source and initial
condition gradients (constant shifts of the hooks)."""
import numpy as np
import pytest

from oracle import adjoint_np as A
from oracle import solver_np as O
from starmap_b200 import configs, starmap_init


def problem(bc=1, substep=True, source=True, shift=(0.0, 0.0, 0.0, 0.0), N=3, n=(6, 7)):
    da, ds, dq, di = shift

    def sig_a(x, y):
        return 0.3 + 0.2 * np.sin(2 * x) * np.cos(y) + da

    prob = dict(name="adj", closure="P", n_mom=N, ax=[-1.0, 1.0, -1.0, 1.0], n=list(n), bc=[bc, bc],
                ic=lambda x, y: np.exp(-8 * (x ** 2 + (y - 0.1) ** 2)) + di, sigma_a=sig_a,
                sigma_s0=lambda x, y: 0.8 + 0.1 * x + ds, tfinal=1e9, t_plot=[0, 1e9], quiet=True)
    if source:
        prob["source"] = lambda x, y: np.exp(-6 * ((x - 0.3) ** 2 + y ** 2)) + dq
    if substep:
        prob.update(filterfunction=configs.exp_filter(2, 3.0), f_position="substep")
    return starmap_init(prob)


def final_state(par, nsteps, U0=None):
    rec = A._Recorder(U0)
    res = O.starmap_solver(par, max_steps=nsteps, advance=rec)
    return res.U


@pytest.mark.parametrize("bc,substep", [(1, True), (0, False)])
def test_oracle_adjoint_dot_product(bc, substep):
    par = problem(bc=bc, substep=substep, source=False)
    nsteps = 4
    shapes = [u.shape for u in final_state(par, 0 + 1)]
    rng = np.random.default_rng(3)
    delta = [rng.standard_normal(s) for s in shapes]
    mu = [rng.standard_normal(s) for s in shapes]
    out = A.adjoint(par, nsteps, lambda U: (mu, 0.0), U0=delta)
    lhs = sum(float(np.sum(u * m)) for u, m in zip(out["U"], mu))
    rhs = sum(float(np.sum(d * l)) for d, l in zip(delta, out["lam0"]))
    assert abs(lhs - rhs) <= 1e-12 * max(abs(lhs), abs(rhs))


def test_oracle_adjoint_matches_central_differences():
    nsteps = 5
    base = problem()
    U = final_state(base, nsteps)
    obs = 0.5 * U[0] + 0.01
    out = A.adjoint(base, nsteps, A.misfit_seed(obs))

    def J(shift):
        Uf = final_state(problem(shift=shift), nsteps)
        return 0.5 * float(np.sum((Uf[0] - obs) ** 2))

    eps = 1e-6
    # sigma_a shifts sA on every grid, hence every sT and sA1
    fd = (J((eps, 0, 0, 0)) - J((-eps, 0, 0, 0))) / (2 * eps)
    ad = sum(float(np.sum(v)) for v in out["g_sT"].values()) + float(np.sum(out["g_sA"]))
    assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)
    # sigma_s0 shifts every sT only
    fd = (J((0, eps, 0, 0)) - J((0, -eps, 0, 0))) / (2 * eps)
    ad = sum(float(np.sum(v)) for v in out["g_sT"].values())
    assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)
    # source of the zeroth moment
    fd = (J((0, 0, eps, 0)) - J((0, 0, -eps, 0))) / (2 * eps)
    ad = float(np.sum(out["g_Q"][0]))
    assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)
    # initial condition of the zeroth moment
    fd = (J((0, 0, 0, eps)) - J((0, 0, 0, -eps))) / (2 * eps)
    ad = float(np.sum(out["lam0"][0]))
    assert abs(fd - ad) <= 1e-6 * abs(fd), (fd, ad)


def test_dexpm1div_branches():
    x = np.array([-1e-5, 1e-4, -0.1, 0.2, -3.0, 2.0])
    h = 1e-6
    num = (O.expm1div(x + h) - O.expm1div(x - h)) / (2 * h)
    got = A.dexpm1div(x)
    # away from the Taylor threshold the derivative of the reference's function
    assert np.allclose(got[2:], num[2:], rtol=1e-7)
    # on the Taylor branch: derivative of 1 + x/2 + x^2/6
    assert np.allclose(got[:2], 0.5 + x[:2] / 3, rtol=0, atol=1e-16)

"""Oracle pins: the reference's own known-answer properties, checked on the CPU
restatements (no GPU).

* P_N == SP_N zeroth moment for isotropic data (starmap_2d_ex_boxes.m:7-16:
  "identical (up to machine accuracy)").
* Mass of the zeroth moment is conserved with sigma_a = 0, no source and
  periodic boundaries (the staggered differences telescope).
* The line source stays symmetric under x <-> y on a square grid.
* The numpy and C restatements agree bit for bit.
"""
import numpy as np
import pytest

import cases
from oracle import c_oracle
from oracle import solver_np as O
from starmap_b200 import configs, starmap_init


def boxes_prob(closure, N, n=40, tfinal=1.0):
    def src(x, y):
        return (((1.75 < x) & (x <= 2.25) & (1.75 < y) & (y <= 2.25)) |
                ((2.75 < x) & (x <= 3.25) & (1.5 < y) & (y <= 2.5))).astype(float) * 2.0
    return dict(closure=closure, n_mom=N, ax=[0, 5, 0, 5], n=[n, n], bc=[1, 1],
                sigma_a=lambda x, y: 0.9, sigma_s0=lambda x, y: 0.1, source=src,
                tfinal=tfinal, t_plot=[0, tfinal], quiet=True)


@pytest.mark.parametrize("N", [3, 5, 9])
def test_pn_equals_spn_for_isotropic_data(N):
    rP = O.starmap_solver(starmap_init(boxes_prob("P", N)))
    rS = O.starmap_solver(starmap_init(boxes_prob("SP", N)))
    a, b = rP.output[0]["U"], rS.output[0]["U"]
    assert rP.step_count == rS.step_count
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()


def test_mass_conservation_void_periodic():
    par = starmap_init(configs.linesource(n=30, n_mom=7, tfinal=1.0))
    r = O.starmap_solver(par)
    X, Y = np.meshgrid(r.output[0]["x"], r.output[0]["y"], indexing="ij")
    m0 = (np.exp(-(X ** 2 + Y ** 2) / (2 * 0.03 ** 2)) / (2 * np.pi * 0.03 ** 2)).sum()
    assert abs(r.output[0]["U"].sum() - m0) <= 1e-13 * m0


def test_linesource_xy_symmetry():
    r = O.starmap_solver(starmap_init(configs.linesource(n=30, n_mom=5, tfinal=1.0)))
    U = r.output[0]["U"]
    assert np.abs(U - U.T).max() <= 1e-13 * np.abs(U).max()


def test_linesource_reflection_symmetry():
    """The line source is symmetric under x -> -x and y -> -y: the zeroth
    moment (cell centres, symmetric about 0) is mirrored in both axes."""
    r = O.starmap_solver(starmap_init(configs.linesource(n=30, n_mom=5, tfinal=1.0)))
    U = np.asarray(r.output[0]["U"])
    scale = np.abs(U).max()
    assert np.abs(U - U[::-1, :]).max() <= 1e-12 * scale
    assert np.abs(U - U[:, ::-1]).max() <= 1e-12 * scale


@pytest.mark.parametrize("name", ["lattice_p5_substep", "box3d_bc1_p2_full", "td_sigma", "spn_3d",
                                  "parabolic_homog", "parabolic_td", "boxes_td_source"])
def test_numpy_and_c_restatements_agree(name):
    par = starmap_init(cases.ALL[name]())
    a = O.starmap_solver(par)
    b = c_oracle.run(par, nthreads=2)
    for u, v in zip(a.output, b.output):
        np.testing.assert_array_equal(u["U"], v["U"])


def test_step_count_overshoot_quirk():
    # dt fixed after the first step; the last step overshoots tfinal (starmap_solver.m:165-208)
    par = starmap_init(configs.linesource(n=100, n_mom=7, tfinal=1.0))
    r = O.starmap_solver(par, max_steps=None)
    assert r.step_count == 67 and r.t > 1.0


def _staggered_l2(U, n, h):
    """Squared discrete L2 norm of one 2D component with the weights of
    starmap_2d_ex_l2norm.m:93-99 (for each axis: a component on the n cell
    centres has end weights 1/2, one on the n+1 faces end weights 0)."""
    U = np.squeeze(np.asarray(U))
    s = [U.shape[d] == n[d] for d in range(2)]
    w1 = np.ones(n[0] + 1 - s[0])
    w1[[0, -1]] = s[0] / 2
    w2 = np.ones(n[1] + 1 - s[1])
    w2[[0, -1]] = s[1] / 2
    return np.prod(h) * w1 @ (U ** 2) @ w2


@pytest.mark.parametrize("bc", [1, 0])
def test_discrete_energy_does_not_grow_in_void(bc):
    """The expanding Gaussian of starmap_2d_ex_l2norm.m (void, all moments at
    output times): the staggered L2 energy never increases and stays within
    2% of its start by t = 0.5."""
    n = 24
    prob = dict(name="gauss", closure="P", n_mom=3, ax=[-1, 1, -1, 1], n=[n, n], bc=[bc, bc],
                ic=lambda x, y, k: (1 / (4 * np.pi * 1e-2)) * np.exp(-(x ** 2 + y ** 2) / (4 * 1e-2)) * (k == 1),
                t_plot=list(np.linspace(0, 0.5, 11)), mom_output="all", output=lambda *a: None, tfinal=0.5,
                quiet=True)
    r = O.starmap_solver(starmap_init(prob), capture_snapshots=True)
    h = [2 / n, 2 / n]
    E = np.array([np.sqrt(sum(_staggered_l2(u, [n, n], h) for u in Us)) for _, Us in r.snapshots])
    assert len(E) == 11
    assert np.all(np.diff(E) <= 1e-14 * E[0])
    assert E[-1] >= 0.98 * E[0]


def test_manufactured_solution_converges_at_second_order():
    """A manufactured solution (the check of starmap_2d_create_mms.m, derived
    by hand here): u_k = e^-t (a_k sin 2piY cos 2piZ + b_k cos 2piY sin 2piZ)
    on the periodic unit square solves u_t + My u_Y + Mz u_Z + sigma_a u = q
    for q built from the closure matrices; the errors at t = 0.25 fall by
    about 4 per halving of h (Y, Z: the solver dimensions of the user's x, y)."""
    N, sa = 3, 0.5
    base = starmap_init(dict(closure="P", n_mom=N, ax=[0, 1, 0, 1], n=[8, 8], bc=[0, 0], quiet=True,
                             ic=lambda x, y: 0 * x, tfinal=0.1))
    My, Mz = np.asarray(base["My"]), np.asarray(base["Mz"])
    n_sys = My.shape[0]
    rng = np.random.default_rng(1)
    a, b = rng.standard_normal(n_sys), rng.standard_normal(n_sys)
    w = 2 * np.pi

    def u(k, Y, Z, t):
        return np.exp(-t) * (a[k] * np.sin(w * Y) * np.cos(w * Z) + b[k] * np.cos(w * Y) * np.sin(w * Z))

    def uY(k, Y, Z, t):
        return np.exp(-t) * w * (a[k] * np.cos(w * Y) * np.cos(w * Z) - b[k] * np.sin(w * Y) * np.sin(w * Z))

    def uZ(k, Y, Z, t):
        return np.exp(-t) * w * (-a[k] * np.sin(w * Y) * np.sin(w * Z) + b[k] * np.cos(w * Y) * np.cos(w * Z))

    def q(x, y, t, k):
        k0 = k - 1
        r = (sa - 1.0) * u(k0, x, y, t)
        for i in range(n_sys):
            r = r + My[k0, i] * uY(i, x, y, t) + Mz[k0, i] * uZ(i, x, y, t)
        return r

    errs = []
    for n in (16, 32, 64):
        par = starmap_init(dict(closure="P", n_mom=N, ax=[0, 1, 0, 1], n=[n, n], bc=[0, 0], quiet=True,
                                ic=lambda x, y, k: u(k - 1, x, y, 0.0), sigma_a=lambda x, y: sa,
                                sigma_s0=lambda x, y: 0.0, source=q, tfinal=0.25))
        r = O.starmap_solver(par)
        err = 0.0
        for k, o in enumerate(r.output):
            X, Y = np.meshgrid(o["x"], o["y"], indexing="ij")
            ex = u(k, X, Y, r.t)
            err = max(err, float(np.sqrt(np.mean((np.asarray(o["U"]).reshape(ex.shape, order="F") - ex) ** 2))))
        errs.append(err)
    rates = np.log2(np.array(errs[:-1]) / np.array(errs[1:]))
    assert np.all(rates > 1.9), rates

"""Time-dependent sources evaluated on the device (``smg_set_source_expr``):
the reference evaluates its source hook on the host before every step
(starmap_solver.m:276-282); here the same function, given as a C++
expression, is evaluated by a kernel before every step, and the loop runs
without host round trips.  Checked against the oracle running the Python
hook: bit for bit where the expression uses only IEEE arithmetic, within
1e-12 where it calls exp/sin (CUDA's and the host's libraries may differ in
the last bit)."""
import numpy as np
import pytest

import cases
from oracle import solver_np as O
from starmap_b200 import _lib, starmap_init
from starmap_b200.solver import starmap_solver

pytestmark = pytest.mark.gpu

MASK_PY = lambda x, y: (((1.75 < x) & (x <= 2.25) & (1.75 < y) & (y <= 2.25)) |
                        ((2.75 < x) & (x <= 3.25) & (1.5 < y) & (y <= 2.50))).astype(np.float64)
MASK_C = ("((((1.75 < x) && (x <= 2.25) && (1.75 < y) && (y <= 2.25)) || "
          "((2.75 < x) && (x <= 3.25) && (1.5 < y) && (y <= 2.50))) ? 1.0 : 0.0)")


def boxes(source, expr, n=20, n_mom=3, tfinal=1.2, **kw):
    p = cases.boxes_td_source()
    p.update(n=[n, n + 3], n_mom=n_mom, tfinal=tfinal, source=source, source_expr=expr, **kw)
    return p


def compare(out, ref, tol):
    for g, r in zip(out, ref):
        if tol == 0:
            np.testing.assert_array_equal(g["U"], r["U"])
        else:
            d = np.linalg.norm((g["U"] - r["U"]).ravel()) / max(np.linalg.norm(r["U"].ravel()), 1e-300)
            assert d <= tol


def test_arithmetic_source_is_bit_identical():
    prob = boxes(lambda x, y, t: (2 + 0.5 * t * t) * MASK_PY(x, y), "(2 + 0.5 * t * t) * " + MASK_C)
    par = starmap_init(prob)
    compare(starmap_solver(par), O.starmap_solver(par).output, 0)


def test_reference_boxes_source_within_tolerance():
    """The boxes example's source, (2 + sin(4 pi t) exp(-t/3)) on two boxes."""
    prob = boxes(cases.boxes_td_source()["source"],
                 "(2 + sin(4 * 3.141592653589793 * t) * exp(-t / 3)) * " + MASK_C)
    par = starmap_init(prob)
    compare(starmap_solver(par), O.starmap_solver(par).output, 1e-12)


def test_source_with_component_and_output_times():
    """A hook taking the component number (source_ind 1..3), output times
    (the loop runs in segments) and a filter."""
    seen = []
    prob = boxes(lambda x, y, t, k: (1.0 + t / k) * MASK_PY(x, y) * (0.5 ** (k - 1)),
                 "(1.0 + t / k) * " + MASK_C + " * pow(0.5, k - 1)", n_mom=4,
                 t_plot=[0.0, 0.4, 1.2], output=lambda par, x, y, U, step: seen.append(step),
                 filterfunction=lambda par, dt, k: np.exp(-0.3 * dt * k ** 2), f_position="substep")
    par = starmap_init(prob)
    assert list(par["source_ind"]) == [1, 2, 3, 4] or len(par["source_ind"]) >= 2
    out = starmap_solver(par)
    ref = O.starmap_solver(par)
    assert seen == [1, 2, 3]
    compare(out, ref.output, 1e-12)


def test_3d_source_expression():
    prob = dict(closure="P", n_mom=2, ax=[-1, 1, -1, 1, -1, 1], n=[9, 8, 7], bc=[1, 0, 1],
                ic=lambda x, y, z: np.exp(-4 * (x * x + y * y + z * z)),
                sigma_a=lambda x, y, z: 0.2, sigma_s0=lambda x, y, z: 1.0,
                source=lambda x, y, z, t: (x + 2 * y - z) * t + 1.0, source_expr="(x + 2 * y - z) * t + 1.0",
                tfinal=0.6, quiet=True)
    par = starmap_init(prob)
    compare(starmap_solver(par), O.starmap_solver(par).output, 0)


def test_device_and_host_source_paths_agree_and_errors():
    """The same run with the source uploaded from the host every step and
    evaluated on the device; a scalar source field and the adjoint are refused."""
    from starmap_b200.solver import setup_gpu
    prob = boxes(lambda x, y, t: (2 + 0.5 * t * t) * MASK_PY(x, y), "(2 + 0.5 * t * t) * " + MASK_C)
    par = starmap_init(prob)
    a = starmap_solver(par)
    prob2 = dict(prob)
    prob2.pop("source_expr")
    b = starmap_solver(starmap_init(prob2))
    compare(a, b, 0)
    S, fs, solver, T = setup_gpu(par)
    try:
        g1 = S.G(1)
        with pytest.raises(_lib.SmgError):   # component 2 has no array source field
            solver.set_source_expr(1, "1.0", [S.xs[g1[0] - 1], S.ys[g1[1] - 1], S.zs[g1[2] - 1]])
        solver.set_state(S.U0)
        solver.set_dt(fs["dt"])
        g = S.G(0)
        solver.set_source_expr(0, "t", [S.xs[g[0] - 1], S.ys[g[1] - 1], S.zs[g[2] - 1]])
        with pytest.raises(_lib.SmgError):
            solver.forward(2, 0)
        solver.set_source_expr(0, None)
        solver.forward(2, 0)
    finally:
        solver.close()


def td_materials(n=18, n_mom=3, tfinal=0.9, **kw):
    """Time-dependent absorption and scattering (cf. the control-rod example:
    a region whose absorption changes in time)."""
    p = dict(name="tdmat", closure="P", n_mom=n_mom, ax=[0, 1, 0, 1], n=[n, n + 2], bc=[0, 1],
             ic=lambda x, y: np.exp(-15 * ((x - .5) ** 2 + (y - .5) ** 2)),
             sigma_a=lambda x, y, t: 0.5 + t * ((x > 0.3) & (x < 0.6)).astype(np.float64) + 0.25 * y,
             sigma_a_expr="0.5 + t * (((x > 0.3) && (x < 0.6)) ? 1.0 : 0.0) + 0.25 * y",
             sigma_s0=lambda x, y, t: 1.0 + 0.5 * t * x, sigma_s0_expr="1.0 + 0.5 * t * x",
             tfinal=tfinal, t_plot=[0, tfinal], quiet=True)
    p.update(kw)
    return p


def test_time_dependent_materials_on_the_device():
    """Materials at t + dt averaged with those at t and the decay factors
    recomputed on the device (CUDA's exp against the host's: 1e-12); the
    last step shortened as the reference does for time-dependent problems."""
    par = starmap_init(td_materials())
    ref = O.starmap_solver(par)
    out = starmap_solver(par)
    compare(out, ref.output, 1e-12)
    assert ref.dts[-1] < ref.dts[0]   # the shortened last step is exercised


def test_time_dependent_materials_with_source_anisotropy_and_output_times():
    seen = []
    prob = td_materials(n_mom=4, t_plot=[0.0, 0.35, 0.9], output=lambda par, x, y, U, step: seen.append(step),
                        sigma_sm=lambda x, y, m, t: 0.1 * 0.5 ** m * (1 + t), sigma_sm_expr="0.1 * pow(0.5, m) * (1 + t)",
                        source=lambda x, y, t: (1 + t) * ((x < 0.2) & (y < 0.2)).astype(np.float64),
                        source_expr="(1 + t) * (((x < 0.2) && (y < 0.2)) ? 1.0 : 0.0)")
    par = starmap_init(prob)
    ref = O.starmap_solver(par)
    out = starmap_solver(par)
    assert seen == [1, 2, 3]
    compare(out, ref.output, 1e-12)


def test_material_expressions_fall_back_without_every_hook():
    """Without an expression for sigma_s0 the host path runs (same result)."""
    prob = td_materials()
    prob.pop("sigma_s0_expr")
    par = starmap_init(prob)
    compare(starmap_solver(par), O.starmap_solver(par).output, 1e-12)


@pytest.mark.parametrize("position", ["substep", "full"])
def test_time_dependent_filter_on_the_device(position):
    """A filter hook taking t (re-evaluated every step: at t - dt/2 and t for
    'substep', at t for 'full'), on the device against the host hook."""
    prob = boxes(lambda x, y, t: (2 + 0.5 * t * t) * MASK_PY(x, y), "(2 + 0.5 * t * t) * " + MASK_C, n_mom=4,
                 filterfunction=lambda par, dt, k, x, y, t: np.exp(-(0.5 + t + 0.1 * x) * dt * (k / 4.0) * (k / 4.0)),
                 filterfunction_expr="exp(-(0.5 + t + 0.1 * x) * dt * (k / 4.0) * (k / 4.0))", f_position=position)
    par = starmap_init(prob)
    compare(starmap_solver(par), O.starmap_solver(par).output, 1e-12)


def test_everything_time_dependent_on_the_device():
    prob = td_materials(n_mom=4, source=lambda x, y, t: (1 + t) * ((x < 0.2) & (y < 0.2)).astype(np.float64),
                        source_expr="(1 + t) * (((x < 0.2) && (y < 0.2)) ? 1.0 : 0.0)",
                        filterfunction=lambda par, dt, k, x, y, t: np.exp(-(1 + t) * dt * (k / 4.0) * (k / 4.0)),
                        filterfunction_expr="exp(-(1 + t) * dt * (k / 4.0) * (k / 4.0))", f_position="substep")
    par = starmap_init(prob)
    compare(starmap_solver(par), O.starmap_solver(par).output, 1e-12)

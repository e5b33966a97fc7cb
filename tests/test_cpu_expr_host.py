"""Host side of the device-evaluated hooks: the time-dependent dt schedule
against the oracle's steps, and the mapping of a user expression's
variables onto the solver dimensions the generated kernels use."""
import pytest

import cases
from oracle import solver_np as O
from starmap_b200 import starmap_init
from starmap_b200.solver import device_source_expr, prepare, td_schedule


@pytest.mark.parametrize("tfinal", [1.5, 0.37])
def test_td_schedule_matches_oracle(tfinal):
    prob = cases.td_sigma()
    prob["tfinal"] = tfinal
    par = starmap_init(prob)
    S = prepare(par)
    ref = O.starmap_solver(par)
    ts, dts = td_schedule(S.dt_hyp, float(par["tfinal"]), float(par["cn"]))
    assert dts == [float(d) for d in ref.dts]
    assert ts[-1] == ref.t


def test_td_schedule_shortens_only_the_last_step():
    ts, dts = td_schedule(0.1, 1.05, 0.9)
    assert all(d == dts[0] for d in dts[:-1]) and dts[-1] < dts[0]
    assert ts[-1] >= 1.05 - 1e-12


def test_expression_variables_map_to_solver_dimensions():
    # 2D: the user's (x, y) are the solver's second and third dimensions
    assert device_source_expr("x * y", 2) == "(y * z)"
    assert device_source_expr("exp(-x*x) + 0x1p-3 * y + 1e-5 * t", 2) == "(exp(-y*y) + 0x1p-3 * z + 1e-5 * t)"
    # 1D: the user's x is the solver's third dimension
    assert device_source_expr("x + t", 1) == "(z + t)"
    # 3D: as written
    assert device_source_expr("x - z", 3) == "(x - z)"
    # a variable the user's hook does not have
    with pytest.raises(ValueError):
        device_source_expr("x + z", 2)
    with pytest.raises(ValueError):
        device_source_expr("y", 1)


@pytest.mark.parametrize("kind,expr", [
    (0, "(2 + sin(4 * 3.141592653589793 * t)) * (x < 0.5 ? 1.0 : 0.0)"),
    (0, "(x + 2 * y - z) * t + 1.0 + k"),
    (0, "0x1.8p+1 * .5e-3 + 1.f - 2E+4"),
    (1, "0.1 * pow(0.5, m) * (1 + t)"),
    (1, "0.5 + t * (((x > 0.3) && (x < 0.6)) ? 1.0 : 0.0) + 0.25 * y"),
    (2, "exp(-(0.5 + t + 0.1 * x) * dt * (k / 4.0) * (k / 4.0))"),
    (2, "fmax(0.0, fmin(1.0, !(k == 0) || true ? 1.0 : 0.0))"),
])
def test_device_expressions_accepted(kind, expr):
    from starmap_b200 import _lib
    assert _lib.lib().smg_check_expr(kind, expr.encode()) == 0


@pytest.mark.parametrize("kind,expr", [
    (0, "Q[0]"),                        # brackets: memory
    (0, "*(double*)0"),                 # type name: pointer cast
    (0, "x; }"),                        # leaving the expression
    (0, "(x = 1.0)"),                   # assignment
    (0, "&x != 0"),                     # address-of
    (0, "C[1] + x"),
    (0, "i0 + x"),                      # kernel locals are not variables
    (1, "m + k"),                       # k is not a material variable
    (2, "x + m"),
    (0, "\"a\""),
    (0, "x)(("),
    (0, "((x)"),
    (0, "1x"),
    (0, ""),
    (3, "x"),                           # unknown kind
])
def test_device_expressions_refused(kind, expr):
    from starmap_b200 import _lib
    L = _lib.lib()
    assert L.smg_check_expr(kind, expr.encode()) == _lib.SMG_EINVAL
    assert L.smg_last_error(None)

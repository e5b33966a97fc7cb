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
    assert device_source_expr("x * y", 2) == "[&](double x, double y) { return (double)(x * y); }(y, z)"
    # 1D: the user's x is the solver's third dimension
    assert device_source_expr("x + t", 1) == "[&](double x) { return (double)(x + t); }(z)"
    # 3D: as written
    assert device_source_expr("x - z", 3) == "(x - z)"

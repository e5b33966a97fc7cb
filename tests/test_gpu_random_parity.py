"""Randomised GPU parity: hypothesis draws small 2D and 3D problems (closure
and order, odd and unequal cell counts, per-axis boundary conditions,
material and source fields, filter position; the generator of
test_cpu_oracle_random.py) and the GPU time loop must reproduce the numpy
oracle bit for bit."""
import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings

from oracle import solver_np as O
from starmap_b200 import starmap_init
from starmap_b200.solver import starmap_solver
from test_cpu_oracle_random import problems

pytestmark = pytest.mark.gpu


@settings(max_examples=12, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(problems())
def test_gpu_matches_oracle_on_random_problems(prob):
    par = starmap_init(prob)
    ref = O.starmap_solver(par)
    out = starmap_solver(par)
    for g, r in zip(out, ref.output):
        np.testing.assert_array_equal(g["U"], r["U"])

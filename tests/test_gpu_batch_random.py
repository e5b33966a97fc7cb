"""Randomised batches: hypothesis draws sets of 2D problems (orders,
closures, odd and unequal sizes, per-axis boundary conditions, fields and
sources, filter '' or 'substep') and the batched solver's family kernels must
reproduce every instance's plain run bit for bit."""
import numpy as np
import pytest
from hypothesis import HealthCheck, given, settings, strategies as st

from starmap_b200 import starmap_init
from starmap_b200.batch import setup_batch
from test_cpu_oracle_random import problems
from test_gpu_batch import plain_reference

pytestmark = pytest.mark.gpu


def _two_d(prob):
    # 2D, and no f_position 'full' (the batch refuses it)
    return len(prob["n"]) == 2 and prob.get("f_position", "") != "full"


@settings(max_examples=6, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow, HealthCheck.filter_too_much])
@given(st.lists(problems().filter(_two_d), min_size=2, max_size=5))
def test_batch_matches_plain_runs_on_random_sets(probs):
    pars = [starmap_init(dict(p, tfinal=1e9)) for p in probs]
    nsteps = 5
    setups, batch = setup_batch(pars)
    try:
        batch.set_states([S.U0 for S, _ in setups])
        batch.set_dt([fs["dt"] for _, fs in setups])
        batch.run(nsteps)
        for i, par in enumerate(pars):
            ref = plain_reference(par, nsteps)
            got = batch.get_state(i)
            for j in ref:
                np.testing.assert_array_equal(got[j], ref[j])
    finally:
        batch.close()

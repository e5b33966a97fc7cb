"""Parabolic time step (par.timestep 1 and 2, starmap_solver.m:168-265,
506-514) with the spectral radius of each trial's growth matrix computed on
the GPU (smg_growth_radius: cuBLAS products, cuSOLVER eigenvalues): the
radius agrees with numpy's eigenvalues of the same matrix, and the search
picks exactly the oracle's dt sequence on the parabolic parity cases."""
import numpy as np
import pytest

import cases
from oracle import solver_np as O
from starmap_b200 import configs, starmap_init, timestep
from starmap_b200.solver import first_step, prepare

from test_cpu_timestep import host_dts

pytestmark = pytest.mark.gpu


@pytest.fixture
def device_eig():
    timestep.use_device_eigenvalues(True)
    yield
    timestep.use_device_eigenvalues(None)


def _radius_both(M, even, odd, decay, dt, ts):
    timestep.use_device_eigenvalues(True)
    g = timestep.growth_factor(M, even, odd, decay, dt, ts)
    timestep.use_device_eigenvalues(False)
    c = timestep.growth_factor(M, even, odd, decay, dt, ts)
    timestep.use_device_eigenvalues(None)
    return g, c


@pytest.mark.parametrize("name,ts", [("parabolic_homog", 1), ("parabolic_homog", 2), ("parabolic_td", 1)])
def test_device_radius_matches_numpy(name, ts):
    prob = cases.ALL[name]()
    prob["timestep"] = ts
    S = prepare(starmap_init(prob))
    fs = first_step(S)
    decay = timestep.decay_vector(S.n_sys, S.gt, S.mom_order, fs["sA"][1, 1, 1], fs["sT"])
    for f in (0.25, 1.0, 3.0, 10.0):
        g, c = _radius_both(S.M_sym, S.even, S.odd, decay, f * S.dt_hyp, ts)
        assert abs(g - c) <= 1e-12 * c, (f, g, c)


def test_device_radius_matches_numpy_p39():
    """The 820-moment lattice system at a few time steps."""
    prob = configs.lattice(n=20)
    prob["timestep"] = 1
    S = prepare(starmap_init(prob))
    fs = first_step(S)
    decay = timestep.decay_vector(S.n_sys, S.gt, S.mom_order, fs["sA"][1, 1, 1], fs["sT"])
    for f in (0.5, 2.0):
        g, c = _radius_both(S.M_sym, S.even, S.odd, decay, f * S.dt_hyp, 1)
        assert abs(g - c) <= 1e-10 * c, (f, g, c)


@pytest.mark.parametrize("name", ["parabolic_homog", "parabolic_td"])
def test_dt_sequence_with_device_eigenvalues_matches_oracle(name, device_eig):
    par = starmap_init(cases.ALL[name]())
    ref = O.starmap_solver(par)
    S, dts = host_dts(par)
    assert dts == [float(d) for d in ref.dts]

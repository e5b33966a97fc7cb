"""The MEX gateway (matlab/starmap_solver_mex.c) without a GPU: it compiles
with -Wall -Wextra -Werror against the header and a test-only stand-in of the
MATLAB C API, links against libstarmap_gpu.so, and turns malformed
descriptors into MATLAB errors (identifier starmap:gpu:*) before any device
work; a well-formed descriptor reaches the library, whose failure here (no
CUDA device) comes back as a starmap:gpu error with the library's message."""
import numpy as np
import pytest

import cases
import mex_gateway as M
from starmap_b200 import starmap_init
from starmap_b200.batch import _tables
from starmap_b200.solver import first_step, handle_tables, prepare


@pytest.fixture(scope="module")
def setup():
    S = prepare(starmap_init(cases.lattice_p5_substep()))
    fs = first_step(S)
    T = _tables(S, fs)
    return M.Gateway(), S, fs, T, handle_tables(S, T)


def _args(G, S, fs, T, tab, overrides=None, U0=None, dt=None, nsteps=3.0):
    d = M.descriptor(G, S, T, tab, overrides)
    U = G.cell([G.array(u) for u in (U0 if U0 is not None else S.U0)])
    return [d, U, G.array(fs["dt"] if dt is None else dt), G.array(nsteps)]


@pytest.mark.parametrize("what,overrides,msg", [
    ("missing field", {"Mx": None}, "descriptor field 'Mx' is missing"),
    ("grid type", {"gt": "bad_gt"}, "'gt' must hold whole numbers in 1..2"),
    ("field number", {"sigma_a": "big"}, "'sigma_a' must hold whole numbers"),
    ("filter mode", {"filter_mode": "three"}, "'filter_mode' must hold whole numbers in 0..2"),
    ("table length", {"source": "short"}, "'source' must have"),
])
def test_malformed_descriptors_raise(setup, what, overrides, msg):
    G, S, fs, T, tab = setup
    ov = {}
    for k, v in overrides.items():
        if v == "bad_gt":
            ov[k] = G.array(np.full((S.n_sys, 3), 3.0))
        elif v == "big":
            ov[k] = G.array(float(len(T.fields) + 5))
        elif v == "three":
            ov[k] = G.array(3.0)
        elif v == "short":
            ov[k] = G.array(np.zeros(S.n_sys - 1))
        else:
            ov[k] = v
    err, out = G.call(_args(G, S, fs, T, tab, ov))
    assert err == "starmap:gpu:desc" and msg in out, (what, err, out)


def test_state_and_usage_errors(setup):
    G, S, fs, T, tab = setup
    bad = [np.zeros(3)] + list(S.U0[1:])
    err, out = G.call(_args(G, S, fs, T, tab, U0=bad))
    assert err == "starmap:gpu:state" and "U0{j}" in out
    err, out = G.call(_args(G, S, fs, T, tab, nsteps=-1.0))
    assert err == "starmap:gpu:usage"
    err, out = G.call(_args(G, S, fs, T, tab)[:3])
    assert err == "starmap:gpu:usage" and "usage" in out


def test_wellformed_descriptor_reaches_the_library(setup):
    """Every descriptor check passes; without a GPU smg_create then fails and
    the gateway reports the library's message."""
    import torch
    if torch.cuda.is_available():
        pytest.skip("a GPU is present: the GPU tests run the gateway")
    G, S, fs, T, tab = setup
    err, out = G.call(_args(G, S, fs, T, tab))
    assert err == "starmap:gpu" and "starmap GPU library" in out


def test_classify_mode_matches_the_library(setup):
    """gt = starmap_solver_mex('classify', Mx, My, Mz): the grid types of
    starmap_solver.m:76-98 as the Python host computes them (smg_classify)."""
    G, S, fs, T, tab = setup
    err, out = G.call([G.string("classify"), G.array(S.Mx), G.array(S.My), G.array(S.Mz)], nlhs=1)
    assert err is None, out
    np.testing.assert_array_equal(G.to_numpy(out[0]), np.asarray(S.gt, dtype=np.float64).reshape(S.n_sys, 3))
    err, out = G.call([G.string("nope"), G.array(S.Mx)], nlhs=1)
    assert err == "starmap:gpu:usage"

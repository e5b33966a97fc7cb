"""The MEX gateway (matlab/starmap_solver_mex.c) on the GPU, called with the
descriptor matlab/starmap_solver.m builds (through a test-only stand-in of
the MATLAB C API): its final components equal the Python drop-in's
starmap_solver output bit for bit on small cases, and at full size the 2D
P39 lattice to t_final = 3.2 matches the oracle's committed digests."""
import numpy as np
import pytest

import cases
import digests
import mex_gateway as M
from starmap_b200 import starmap_init
from starmap_b200.batch import _tables
from starmap_b200.solver import first_step, handle_tables, prepare, starmap_solver, step_times

pytestmark = pytest.mark.gpu


def run_gateway(G, prob):
    par = starmap_init(prob)
    S = prepare(par)
    fs = first_step(S)
    T = _tables(S, fs)
    nsteps = len(step_times(fs["dt"], float(S.par["tfinal"])))
    d = M.descriptor(G, S, T, handle_tables(S, T))
    U0 = G.cell([G.array(u) for u in S.U0])
    err, out = G.call([d, U0, G.array(fs["dt"]), G.array(float(nsteps))])
    assert err is None, out
    U = [G.to_numpy(G.L.mxGetCell(out[0], j)) for j in range(S.n_sys)]
    ms = G.to_numpy(out[1]).item()
    return S, U, ms, nsteps


@pytest.mark.parametrize("name", ["lattice_p5_substep", "lattice_p4_full", "lin_p7_periodic", "odd_mixed_bc",
                                  "aniso_2d", "pt3d_p3", "box3d_bc1_p2_full", "spn_2d"])
def test_gateway_matches_python_drop_in(name):
    G = M.Gateway()
    prob = dict(cases.ALL[name]())
    prob["mom_output"] = "all"
    S, U, ms, nsteps = run_gateway(G, prob)
    out = starmap_solver(starmap_init(prob))
    assert ms > 0 and len(out) == S.n_sys
    for j in range(S.n_sys):
        a = np.asarray(U[j]).ravel(order="F")
        b = np.asarray(out[j]["U"]).ravel(order="F")
        assert a.shape == b.shape and np.count_nonzero(a != b) == 0, (name, j)


def test_gateway_full_size_lattice_matches_oracle_digests():
    G = M.Gateway()
    prob, _ = digests.full_size_prob("c2_lattice_p39_350")
    S, U, ms, nsteps = run_gateway(G, prob)
    ref = digests.load("c2_lattice_p39_350")
    assert nsteps == ref["steps"] == 321
    # the output struct's 2D layout (starmap_solver.m:484-500)
    comps = [U[j].reshape(len(S.ys[S.G(j)[1] - 1]), -1, order="F") for j in range(S.n_sys)]
    bad = digests.compare(digests.state_digest(comps), ref["components"])
    assert not bad, bad[:3]

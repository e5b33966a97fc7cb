"""Parabolic time-step selection (``par.timestep`` 1 and 2,
starmap_solver.m:168-265, 506-514): the host implementation in
``starmap_b200.timestep`` against the oracle's restatement, and the
properties of the selected step."""
import numpy as np
import pytest

import cases
from oracle import solver_np as O
from starmap_b200 import starmap_init, timestep
from starmap_b200.solver import first_step, prepare, step_materials


def host_dts(par):
    """dt of every step as the host loop of ``starmap_solver`` chooses it."""
    S = prepare(par)
    fs = first_step(S)
    dt, sA, sT = fs["dt"], fs["sA"], fs["sT"]
    tfinal = float(par["tfinal"])
    dts = [dt]
    t = dt
    while t < tfinal:
        if S.time_dependent.any():
            dt, sA, sT, _, _ = step_materials(S, t, dt, sA, sT)
        t = t + dt
        dts.append(dt)
    return S, dts


@pytest.mark.parametrize("name", ["parabolic_homog", "parabolic_td"])
def test_dt_sequence_matches_oracle(name):
    par = starmap_init(cases.ALL[name]())
    ref = O.starmap_solver(par)
    S, dts = host_dts(par)
    assert dts == [float(d) for d in ref.dts]
    # the parabolic step is longer than the hyperbolic one for these materials
    assert min(dts[:-1]) > S.dt_hyp * float(par["cn"])


@pytest.mark.parametrize("ts", [1, 2])
def test_selected_step_is_stable(ts):
    prob = cases.parabolic_homog()
    prob["timestep"] = ts
    S = prepare(starmap_init(prob))
    fs = first_step(S)
    cn = float(S.par["cn"])
    tleft = float(S.par["tfinal"]) / cn
    decay = timestep.decay_vector(S.n_sys, S.gt, S.mom_order, fs["sA"][1, 1, 1], fs["sT"])
    dt_b, la0 = timestep.search(S.M_sym, S.even, S.odd, decay, 0.0, S.dt_hyp, tleft, ts)
    assert fs["dt"] == min(dt_b, tleft) * cn
    assert timestep.growth_factor(S.M_sym, S.even, S.odd, decay, dt_b, ts) < la0
    # doubling the step leaves the stable region
    assert timestep.growth_factor(S.M_sym, S.even, S.odd, decay, 2 * dt_b, ts) >= la0


def test_relative_stability_allows_no_longer_step():
    """timestep 2 measures growth relative to exp(-sigma_a dt), which can only
    raise the growth factor: the selected step is no longer than with 1."""
    a, b = cases.parabolic_homog(), cases.parabolic_homog()
    b["timestep"] = 2
    da = first_step(prepare(starmap_init(a)))["dt"]
    db = first_step(prepare(starmap_init(b)))["dt"]
    assert db <= da


def test_growth_factor_matches_oracle():
    par = starmap_init(cases.parabolic_td())
    S = prepare(par)
    fs = first_step(S)
    decay = timestep.decay_vector(S.n_sys, S.gt, S.mom_order, fs["sA"][1, 1, 1], fs["sT"])
    c, *_ = O._classify(S.Mx, S.My, S.Mz)
    Msym = -1j * (S.Mx / S.h[0] + S.My / S.h[1] + S.Mz / S.h[2])
    for dt in (0.01, 0.05, 0.2):
        for ts in (1, 2):
            a = timestep.growth_factor(S.M_sym, S.even, S.odd, decay, dt, ts)
            b = O._growth_factor(Msym, c, decay, dt, ts)
            assert abs(a - b) <= 1e-13 * b


def test_fallback_to_materials_at_t_when_average_unstable(monkeypatch):
    """With the averaged materials unstable, the step uses those at time t
    (starmap_solver.m:260-264)."""
    par = starmap_init(cases.parabolic_td())
    S = prepare(par)
    fs = first_step(S)
    monkeypatch.setattr(timestep, "stable", lambda *a: False)
    dt, sA, sT, sA1, sT1 = step_materials(S, fs["dt"], fs["dt"], fs["sA"], fs["sT"])
    assert np.array_equal(sA1, fs["sA"][1, 1, 1])
    assert all(np.array_equal(sT1[k], fs["sT"][k]) for k in S.sg)


def test_3d_field_with_planes_is_rejected():
    """min(min(.)) of a 3D field leaves a vector, which the reference cannot
    store in the decay vector; the host stops the same way."""
    prob = cases.pt3d_p3()
    prob["timestep"] = 1
    prob["sigma_s0"] = lambda x, y, z: 1.0 + 0.1 * z
    with pytest.raises(ValueError):
        first_step(prepare(starmap_init(prob)))


def test_search_with_zero_cross_sections_and_little_time_left():
    """sigma = 0: below the stability limit the growth factor is 1, so the
    search lowers its threshold to 1 and still brackets the limit; with less
    time left than a step, the lower end stops at or past the time left."""
    prob = cases.parabolic_homog()
    prob["sigma_a"] = lambda x, y: 0.0
    prob["sigma_s0"] = lambda x, y: 0.0
    S = prepare(starmap_init(prob))
    decay = np.zeros(S.n_sys)
    dt_b, la0 = timestep.search(S.M_sym, S.even, S.odd, decay, 0.0, S.dt_hyp, 1e9, 1)
    assert 0 < dt_b < 1e9
    assert timestep.growth_factor(S.M_sym, S.even, S.odd, decay, dt_b, 1) < la0
    # the hyperbolic step is stable, so with less time left than it the
    # bracket never moves: its lower end stays at dt_hyp (the caller then
    # takes min(dt, time left) * cn)
    small = 0.1 * S.dt_hyp
    dt_s, _ = timestep.search(S.M_sym, S.even, S.odd, decay, 0.0, S.dt_hyp, small, 1)
    assert dt_s == S.dt_hyp
    assert dt_b >= S.dt_hyp


from hypothesis import HealthCheck, given, settings, strategies as st  # noqa: E402


@settings(max_examples=12, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(ts=st.sampled_from([0, 1, 2]), n=st.integers(4, 8), a0=st.floats(0.5, 4.0), a1=st.floats(0.0, 2.0),
       w=st.floats(0.5, 8.0), s0=st.floats(0.0, 4.0), tfinal=st.floats(0.05, 0.4))
def test_host_dt_sequence_matches_oracle_on_random_td_problems(ts, n, a0, a1, w, s0, tfinal):
    """Time-dependent absorption with the hyperbolic or a parabolic step: the
    host loop's dt of every step equals the oracle's."""
    prob = dict(name="td", closure="P", n_mom=2, timestep=ts, ax=[0, 1, 0, 1], n=[n, n + 1], bc=[0, 1],
                ic=lambda x, y: np.exp(-10 * ((x - .5) ** 2 + (y - .5) ** 2)),
                sigma_a=lambda x, y, t: a0 + a1 * np.sin(w * t) + 0 * x, sigma_s0=lambda x, y: s0 + 0 * x,
                tfinal=tfinal, quiet=True)
    par = starmap_init(prob)
    ref = O.starmap_solver(par)
    _, dts = host_dts(par)
    assert dts == [float(d) for d in ref.dts]

"""Batched solver: every instance bit-identical to its own plain run; the
bounded grid barrier reports a timeout without hanging; the autotuner keeps
the state."""
import numpy as np
import pytest

from starmap_b200 import configs, starmap_init
from starmap_b200._lib import SmgError, SMG_ETIMEOUT
from starmap_b200.batch import BARRIER_EXTRA, JIT, PERSISTENT, SPIN_LIMIT, STEPS_PER_LAUNCH, setup_batch
from starmap_b200.solver import setup_gpu

pytestmark = pytest.mark.gpu


def small_batch(n=6, seed=7):
    probs = configs.batched_sweep(n_inst=n, seed=seed, edges=(16, 24, 32), orders=(1, 3, 5, 7))
    return [starmap_init(p) for p in probs]


def plain_reference(par, nsteps):
    S, fs, solver, T = setup_gpu(par)
    try:
        solver.set_state(S.U0)
        solver.set_dt(fs["dt"])
        solver.run(nsteps)
        return solver.get_state()
    finally:
        solver.close()


@pytest.mark.parametrize("spl", [0, 1, 4, 8])
def test_batch_matches_plain_runs(spl):
    """spl = steps per persistent launch; 0 = one launch per phase."""
    pars = small_batch()
    nsteps = 13
    setups, batch = setup_batch(pars)
    try:
        batch.tune(JIT, 0)   # the precompiled kernels
        if spl == 0:
            batch.tune(PERSISTENT, 0)
        else:
            batch.tune(STEPS_PER_LAUNCH, spl)
        batch.set_states([S.U0 for S, _ in setups])
        batch.set_dt([fs["dt"] for _, fs in setups])
        batch.run(nsteps)
        ms, launches = batch.last_run_stats()
        assert launches == (2 * nsteps + 1 if spl == 0 else -(-nsteps // spl))
        for i, par in enumerate(pars):
            ref = plain_reference(par, nsteps)
            got = batch.get_state(i)
            for j in ref:
                np.testing.assert_array_equal(got[j], ref[j])
    finally:
        batch.close()


def test_batch_family_kernels_match_plain_runs():
    """Generated family kernels (the default): instances of equal structure and
    different grids share kernels; every instance bit-identical to its plain run."""
    probs = configs.batched_sweep(n_inst=10, seed=11, edges=(16, 24, 33, 40), orders=(1, 3, 5))
    for p in probs[::2]:
        p["bc"] = [1, 1]   # extrapolation boundaries: staggered extents differ from the cell counts
    pars = [starmap_init(p) for p in probs]
    nsteps = 9
    setups, batch = setup_batch(pars)
    try:
        batch.set_states([S.U0 for S, _ in setups])
        batch.set_dt([fs["dt"] for _, fs in setups])
        batch.run(nsteps)
        used, fams = batch.info()
        # at least one family per (order, boundary condition); instances whose
        # spacings need different division forms fall into different ones
        structures = {(int(p["n_mom"]), tuple(int(b) for b in p["bc"])) for p in pars}
        assert used and len(structures) <= fams <= len(pars)
        for i, par in enumerate(pars):
            ref = plain_reference(par, nsteps)
            got = batch.get_state(i)
            for j in ref:
                np.testing.assert_array_equal(got[j], ref[j])
        # a second run replays the captured graph with fresh geometry and state
        batch.set_states([S.U0 for S, _ in setups])
        batch.run(nsteps)
        got = batch.get_state(3)
        ref = plain_reference(pars[3], nsteps)
        for j in ref:
            np.testing.assert_array_equal(got[j], ref[j])
    finally:
        batch.close()


def test_batch_barrier_timeout_is_reported_and_recoverable():
    pars = small_batch(n=3)
    setups, batch = setup_batch(pars)
    try:
        batch.tune(JIT, 0)   # the persistent kernel's grid barrier
        batch.set_states([S.U0 for S, _ in setups])
        batch.set_dt([fs["dt"] for _, fs in setups])
        batch.tune(SPIN_LIMIT, 20000)
        batch.tune(BARRIER_EXTRA, 1)      # the barrier waits for a CTA that does not exist
        with pytest.raises(SmgError) as ei:
            batch.run(2)
        assert ei.value.code == SMG_ETIMEOUT
        batch.tune(BARRIER_EXTRA, 0)
        batch.tune(SPIN_LIMIT, 1 << 25)
        batch.set_states([S.U0 for S, _ in setups])
        batch.run(5)                      # the context is still usable
        ref = plain_reference(pars[0], 5)
        got = batch.get_state(0)
        for j in ref:
            np.testing.assert_array_equal(got[j], ref[j])
    finally:
        batch.close()


def test_batch_autotune_restores_state():
    pars = small_batch(n=4, seed=3)
    setups, batch = setup_batch(pars)
    try:
        batch.set_states([S.U0 for S, _ in setups])
        batch.set_dt([fs["dt"] for _, fs in setups])
        best = batch.autotune(probe_steps=2)
        assert best > 0
        cfg = batch.config()
        assert cfg["block"] in (64, 128) and cfg["group"] in (4, 8, 16) and cfg["grid"] >= 0
        batch.run(7)
        for i, par in enumerate(pars):
            ref = plain_reference(par, 7)
            got = batch.get_state(i)
            for j in ref:
                np.testing.assert_array_equal(got[j], ref[j])
    finally:
        batch.close()


def test_batch_refuses_device_expressions():
    """A batch advances its instances with its own kernels, which do not
    evaluate smg_set_source_expr expressions: such an instance is refused."""
    from starmap_b200 import _lib
    probs = configs.batched_sweep(n_inst=2, seed=5, edges=(16,), orders=(1,))
    for p in probs:
        p["source"] = lambda x, y: 0.1 * x   # an array source field on component 1
    pars = [starmap_init(p) for p in probs]
    setups, batch = setup_batch(pars)
    try:
        batch.set_states([S.U0 for S, _ in setups])
        batch.set_dt([fs["dt"] for _, fs in setups])
        S0 = setups[0][0]
        g = S0.G(0)
        batch.inst[0].set_source_expr(0, "t", [S0.xs[g[0] - 1], S0.ys[g[1] - 1], S0.zs[g[2] - 1]])
        with pytest.raises(_lib.SmgError):
            batch.run(2)
        batch.inst[0].set_source_expr(0, None)
        batch.run(2)
    finally:
        batch.close()

"""GPU time loop vs the CPU oracle on identical inputs (bar: 1e-12 relative L2
per moment at t_final; the arithmetic is mirrored, so results are expected to
be bit-identical and that is asserted too)."""
import numpy as np
import pytest

import cases
from oracle import solver_np as O
from starmap_b200 import starmap_init
from starmap_b200.solver import starmap_solver

pytestmark = pytest.mark.gpu
REL_L2_TOL = 1e-12


def rel_l2(a, b):
    nb = np.linalg.norm(b.ravel())
    return np.linalg.norm((a - b).ravel()) / (nb if nb > 0 else 1.0)


def compare(out_gpu, out_ref):
    assert len(out_gpu) == len(out_ref)
    worst = 0.0
    mism = 0
    for g, r in zip(out_gpu, out_ref):
        assert g["U"].shape == r["U"].shape
        for key in ("x", "y", "z"):
            if key in r:
                np.testing.assert_array_equal(g[key], r[key])
        worst = max(worst, rel_l2(g["U"], r["U"]))
        mism += int(np.count_nonzero(g["U"] != r["U"]))
    return worst, mism


VARIANTS = {"auto": 0, "generic": 1, "strip": 2, "staged": 3, "pair": 4, "jit": 5}


@pytest.mark.parametrize("variant", sorted(VARIANTS))
@pytest.mark.parametrize("name", sorted(cases.ALL))
def test_parity_small(name, variant, monkeypatch):
    from starmap_b200 import solver as solver_mod
    monkeypatch.setattr(solver_mod, "DEFAULT_VARIANT", VARIANTS[variant])
    par = starmap_init(cases.ALL[name]())
    ref = O.starmap_solver(par)
    out = starmap_solver(par)
    worst, mism = compare(out, ref.output)
    assert worst <= REL_L2_TOL, f"{name}: worst relative L2 {worst:.3e}"
    assert mism == 0, f"{name}: {mism} values differ from the oracle (worst rel L2 {worst:.3e})"


def test_program_cache_keys_on_every_generator_input():
    """Generated programs are shared between handles of one process when
    their generator inputs are equal.  Problems that differ only in the grid
    spacing, the boundary conditions, the closure (coupling weights), the
    filter position or the array-ness of a coefficient get programs of their
    own: in one process, alternating between them, each matches the oracle
    bit for bit."""
    base = cases.lattice_p5_substep()
    probs = [base,
             dict(base, ax=[0.0, 9.0, 0.0, 9.0]),                 # spacing
             dict(base, bc=[0, 0]),                                # boundary conditions
             dict(base, closure="SP"),                             # coupling weights
             dict(base, f_position="full"),                        # filter
             dict(base, sigma_s0=lambda x, y: 1.0)]                # an array coefficient becomes a scalar
    for prob in probs + probs[::-1]:
        par = starmap_init(dict(prob))
        ref = O.starmap_solver(par)
        out = starmap_solver(par)
        worst, mism = compare(out, ref.output)
        assert mism == 0, f"{mism} values differ from the oracle (worst rel L2 {worst:.3e})"


def test_output_times_and_callback():
    """t_plot interpolation and the output hook (starmap_solver.m:425-473)."""
    prob = cases.lattice_p5_substep()
    prob["t_plot"] = [0.0, 0.7, 1.3, 2.0, 5.0]
    prob["mom_output"] = "all"
    seen = []

    def output(par, x, y, U, step):
        seen.append((step, [u.copy() for u in U]))

    prob["output"] = output
    par = starmap_init(prob)
    ref = O.starmap_solver(par, capture_snapshots=True)
    starmap_solver(par)
    assert len(seen) == len(ref.snapshots) == 5
    for (step, Ug), (tp, Ur) in zip(seen, ref.snapshots):
        for ug, ur in zip(Ug, Ur):
            ur2 = ur.reshape(ug.shape, order="F")
            assert rel_l2(ug, ur2) <= REL_L2_TOL


def test_snapshot_interpolation_on_device():
    """smg_snapshot / smg_get_interp: (1 - lam) * snapshot + lam * state in
    the host's operation order, for small and for split (larger than the
    staging buffer) components."""
    from starmap_b200.solver import GpuSolver, prepare
    for prob in (cases.box3d_bc1_p2_full(),
                 dict(closure="P", n_mom=1, ax=[-1, 1, -1, 1, -1, 1], n=[265, 264, 263], bc=[1, 0, 1],
                      ic=lambda x, y, z: 0 * x, sigma_a=lambda x, y, z: 0.0, sigma_s0=lambda x, y, z: 1.0,
                      tfinal=1.0, quiet=True)):
        S = prepare(starmap_init(prob))
        rng = np.random.default_rng(3)
        fields = [(0.3, (1, 1, 1)), (1.0, (1, 1, 1))]
        solver = GpuSolver(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, fields, [0] * S.n_sys, 0, [-1] * S.n_sys,
                           decay_t=[1] * S.n_sys, decay_a=1)
        try:
            A = [rng.standard_normal(solver.extents(j)) for j in range(S.n_sys)]
            B = [rng.standard_normal(solver.extents(j)) for j in range(S.n_sys)]
            solver.set_state(A)
            solver.snapshot()
            solver.set_state(B)
            for lam in (0.0, 0.3, 1.0, 0.7071):
                got = solver.get_interp(lam, [0, S.n_sys - 1])
                for j in (0, S.n_sys - 1):
                    np.testing.assert_array_equal(got[j], (1 - lam) * A[j] + lam * B[j])
        finally:
            solver.close()


def test_all_moments_at_output_times():
    """mom_output 'all' with several output times inside steps: the device
    interpolation gives the oracle's snapshots bit for bit."""
    prob = cases.lattice_p5_substep()
    prob["t_plot"] = [0.0, 0.33, 0.7, 1.45, 2.0]
    prob["mom_output"] = "all"
    seen = []
    prob["output"] = lambda par, x, y, U, step: seen.append([u.copy() for u in U])
    par = starmap_init(prob)
    ref = O.starmap_solver(par, capture_snapshots=True)
    starmap_solver(par)
    assert len(seen) == len(ref.snapshots) == 5
    for Ug, (tp, Ur) in zip(seen, ref.snapshots):
        for ug, ur in zip(Ug, Ur):
            np.testing.assert_array_equal(ug, ur.reshape(ug.shape, order="F"))


def test_state_roundtrip_and_layout():
    """Upload/download through the C ABI is the identity on every component."""
    from starmap_b200.solver import GpuSolver, prepare
    par = starmap_init(cases.box3d_bc1_p2_full())
    S = prepare(par)
    rng = np.random.default_rng(7)
    fields = [(0.3, (1, 1, 1)), (1.0, (1, 1, 1))]
    solver = GpuSolver(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, fields, [0] * S.n_sys, 0, [-1] * S.n_sys,
                       decay_t=[1] * S.n_sys, decay_a=1)
    try:
        U = [rng.standard_normal(solver.extents(j)) for j in range(S.n_sys)]
        solver.set_state(U)
        back = solver.get_state()
        for j in range(S.n_sys):
            np.testing.assert_array_equal(back[j], U[j])
        nbytes, dims = solver.layout()
        assert dims[0] % 8 == 0 and dims[3] % 32 == 0 and nbytes > 0
        assert solver.check_finite() == 0
    finally:
        solver.close()


@pytest.mark.parametrize("which", ["many_components", "large_components"])
def test_state_transfer_paths(which):
    """The staged transfers: 820 components of 80 KB (chunks bounded by the
    64-component kernel limit and by the staging size), and 3D components of
    150 MB, larger than the staging buffer, which take the pitched copy.
    Upload then download is the identity, and a partial download returns
    only the components asked for."""
    from starmap_b200 import configs
    from starmap_b200.solver import GpuSolver, prepare
    if which == "many_components":
        par = starmap_init(configs.lattice(n=100, n_mom=39))
    else:
        par = starmap_init(dict(closure="P", n_mom=1, ax=[-1, 1, -1, 1, -1, 1], n=[265, 264, 263], bc=[1, 0, 1],
                                ic=lambda x, y, z: 0 * x, sigma_a=lambda x, y, z: 0.0,
                                sigma_s0=lambda x, y, z: 1.0, tfinal=1.0, quiet=True))
    S = prepare(par)
    rng = np.random.default_rng(11)
    fields = [(0.3, (1, 1, 1)), (1.0, (1, 1, 1))]
    solver = GpuSolver(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, fields, [0] * S.n_sys, 0, [-1] * S.n_sys,
                       decay_t=[1] * S.n_sys, decay_a=1)
    try:
        U = [rng.standard_normal(solver.extents(j)) for j in range(S.n_sys)]
        if which == "large_components":
            assert U[0].nbytes > 64 << 20
        solver.set_state(U)
        back = solver.get_state()
        for j in range(S.n_sys):
            np.testing.assert_array_equal(back[j], U[j])
        some = solver.get_state(which=[0, S.n_sys - 1])
        assert sorted(some) == [0, S.n_sys - 1]
        np.testing.assert_array_equal(some[S.n_sys - 1], U[S.n_sys - 1])
    finally:
        solver.close()


def test_full_size_lattice_prefix_vs_c_oracle():
    """The benchmark workload at full size (820 moments, 350x350) for a prefix
    of 4 steps, GPU (default fused strip kernels) vs the oracle's C restatement."""
    from oracle import c_oracle
    from starmap_b200 import configs
    from starmap_b200.solver import setup_gpu
    par = starmap_init(configs.lattice())
    nsteps = 4
    ref = c_oracle.run(par, max_steps=nsteps)
    S, fs, solver, T = setup_gpu(par)
    try:
        solver.set_state(S.U0)
        solver.set_dt(fs["dt"])
        solver.run(nsteps)
        U = solver.get_state()
    finally:
        solver.close()
    worst = 0.0
    mism = 0
    for j in range(S.n_sys):
        r = ref.U[j]
        worst = max(worst, rel_l2(U[j], r))
        mism += int(np.count_nonzero(U[j] != r))
    assert ref.step_count == nsteps
    assert worst <= REL_L2_TOL
    assert mism == 0


def test_variants_agree_on_c1_linesource():
    """Line source P7 100x100 to t=1 (67 steps): all kernel variants bit-identical."""
    from starmap_b200 import configs
    from starmap_b200.solver import setup_gpu
    par = starmap_init(configs.linesource())
    outs = []
    for v in (0, 1, 2, 3, 4, 5):
        S, fs, solver, T = setup_gpu(par)
        try:
            solver.set_variant(v)
            solver.set_state(S.U0)
            solver.set_dt(fs["dt"])
            solver.run(67)
            outs.append(solver.get_state())
        finally:
            solver.close()
    for j in outs[0]:
        np.testing.assert_array_equal(outs[0][j], outs[1][j])
        np.testing.assert_array_equal(outs[0][j], outs[2][j])
        np.testing.assert_array_equal(outs[0][j], outs[3][j])
        np.testing.assert_array_equal(outs[0][j], outs[4][j])
        np.testing.assert_array_equal(outs[0][j], outs[5][j])


def test_auto_runs_the_specialised_kernels():
    """On a B200 with NVRTC, AUTO compiles and runs the generated kernels."""
    from starmap_b200 import configs
    from starmap_b200.solver import setup_gpu
    par = starmap_init(configs.linesource())
    S, fs, solver, T = setup_gpu(par)
    try:
        solver.set_state(S.U0)
        solver.set_dt(fs["dt"])
        solver.run(3)
        v, why = solver.active_variant()
    finally:
        solver.close()
    assert v == 5, why


@pytest.mark.parametrize("block,group,split,calls,xpair,prefetch", [
    (32, 1, 4, 0, 0, 0), (128, 3, 1, 1, 0, 0), (256, 64, 4, 0, 1, 0), (64, 4, 0, 0, 1, 0), (64, 2, 3, 1, 1, 0),
    (64, 8, 16, 0, 0, 1), (64, 8, 16, 0, 2, 0), (32, 3, 16, 0, 2, 0)])
@pytest.mark.parametrize("band,const", [(0, 0), (3, 0), (0, 1)])
def test_jit_tuning_keeps_results(block, group, split, calls, xpair, prefetch, band, const):
    from starmap_b200 import _lib
    from starmap_b200.solver import setup_gpu
    par = starmap_init(cases.odd_mixed_bc())
    outs = []
    for tune in (False, True):
        S, fs, solver, T = setup_gpu(par)
        try:
            if tune:
                solver.tune(_lib.SMG_TUNE_JIT_BLOCK, block)
                solver.tune(_lib.SMG_TUNE_JIT_GROUP, group)
                solver.tune(_lib.SMG_TUNE_JIT_SPLIT, split)
                solver.tune(_lib.SMG_TUNE_JIT_CALLS, calls)
                solver.tune(_lib.SMG_TUNE_JIT_XPAIR, xpair)
                solver.tune(_lib.SMG_TUNE_JIT_PREFETCH, prefetch)
                solver.tune(_lib.SMG_TUNE_JIT_BAND, band)
                solver.tune(_lib.SMG_TUNE_JIT_CONST, const)
                solver.tune(_lib.SMG_TUNE_JIT_LANES, group % 3)   # 0 (all), 1 or 2 kernels at a time
                solver.set_variant(5)
            else:
                solver.set_variant(4)
            solver.set_state(S.U0)
            solver.set_dt(fs["dt"])
            solver.run(7)
            outs.append(solver.get_state())
        finally:
            solver.close()
    for j in outs[0]:
        np.testing.assert_array_equal(outs[0][j], outs[1][j])


@pytest.mark.parametrize("name", ["lattice_p5_substep", "pt3d_p3", "box3d_bc1_p2_full"])
def test_graph_steps_keep_results(name):
    """Direct launches, graphs of 1, 5 and 64 steps and the default policy
    give bit-identical states (the block boundaries split the fused A-A
    phases, which must not change a value)."""
    from starmap_b200 import _lib
    from starmap_b200.solver import setup_gpu
    par = starmap_init(cases.ALL[name]())
    outs = []
    for gb in (-1, 0, 1, 5, 64):
        S, fs, solver, T = setup_gpu(par)
        try:
            solver.tune(_lib.SMG_TUNE_GRAPH_STEPS, gb)
            solver.set_state(S.U0)
            solver.set_dt(fs["dt"])
            solver.run(70)
            solver.run(11)
            outs.append(solver.get_state())
        finally:
            solver.close()
    for o in outs[1:]:
        for j in outs[0]:
            np.testing.assert_array_equal(outs[0][j], o[j])


def test_jit_band_order_keeps_results_3d():
    """CTA order by bands of rows (the default for component slots of 4 MB and
    more: here 84^3 cells, about 714-row bands) against group-major order and
    explicit odd band sizes: bit-identical states."""
    from starmap_b200 import _lib, configs
    from starmap_b200.solver import setup_gpu
    par = starmap_init(configs.pointsource3d(n=84, n_mom=9, tfinal=0.1))
    outs = []
    for band in (-1, 0, 1, 333):
        S, fs, solver, T = setup_gpu(par)
        try:
            solver.tune(_lib.SMG_TUNE_JIT_BAND, band)
            solver.set_variant(5)
            solver.set_state(S.U0)
            solver.set_dt(fs["dt"])
            solver.run(4)
            outs.append(solver.get_state([0, 7, 50, 99]))
        finally:
            solver.close()
    for o in outs[1:]:
        for j in outs[0]:
            np.testing.assert_array_equal(outs[0][j], o[j])


def test_gpu_pn_equals_spn_boxes():
    from test_cpu_oracle_properties import boxes_prob
    outP = starmap_solver(starmap_init(boxes_prob("P", 9)))
    outS = starmap_solver(starmap_init(boxes_prob("SP", 9)))
    a, b = outP[0]["U"], outS[0]["U"]
    assert np.abs(a - b).max() <= 1e-12 * np.abs(a).max()


def test_full_size_linesource_properties():
    """2D P7 line source at full size (100x100, t=1, 67 steps): mass of the
    zeroth moment conserved, x<->y symmetric, all moments finite."""
    from starmap_b200 import configs
    out = starmap_solver(starmap_init(configs.linesource()))
    U = out[0]["U"]
    X, Y = np.meshgrid(out[0]["x"], out[0]["y"], indexing="ij")
    m0 = (np.exp(-(X ** 2 + Y ** 2) / (2 * 0.03 ** 2)) / (2 * np.pi * 0.03 ** 2)).sum()
    assert abs(U.sum() - m0) <= 1e-12 * m0
    assert np.abs(U - U.T).max() <= 1e-12 * np.abs(U).max()
    assert all(np.isfinite(o["U"]).all() for o in out)


def test_state_sumsq_reduction():
    """Per-component sums of squares of the state (deterministic two-pass
    reduction through the handle's scratch) against the host sum."""
    from starmap_b200.solver import GpuSolver, prepare
    par = starmap_init(cases.box3d_bc1_p2_full())
    S = prepare(par)
    rng = np.random.default_rng(11)
    fields = [(0.3, (1, 1, 1)), (1.0, (1, 1, 1))]
    solver = GpuSolver(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, fields, [0] * S.n_sys, 0, [-1] * S.n_sys,
                       decay_t=[1] * S.n_sys, decay_a=1)
    try:
        U = [rng.standard_normal(solver.extents(j)) for j in range(S.n_sys)]
        solver.set_state(U)
        a = solver.state_sumsq()
        b = solver.state_sumsq()
        np.testing.assert_array_equal(a, b)
        ref = np.array([np.sum(u * u) for u in U])
        assert np.max(np.abs(a - ref) / ref) <= 1e-13
    finally:
        solver.close()


STAGED_CASES = ["lattice_p5_substep", "lattice_p4_full", "lattice_p6_nofilter", "odd_mixed_bc", "aniso_2d",
                "lin_p7_periodic", "spn_2d", "pt3d_p3", "box3d_bc1_p2_full", "spn_3d"]


@pytest.mark.parametrize("shape", [(1, 4, 3, 0), (1, 1, 2, 1), (1, 3, 6, 5), (2, 4, 3, 0), (2, 1, 2, 1), (2, 3, 6, 5),
                                   (2, 8, 2, 0), (2, 16, 4, 0), (3, 4, 3, 0), (0, 4, 3, 0)])
@pytest.mark.parametrize("name", STAGED_CASES)
def test_staged_kernels_vs_oracle(name, shape):
    """The generated kernels in the staged forms (row segments copied into a
    shared-memory ring by the bulk copy engine, or by the consumer warps' own
    asynchronous copies), with a per-thread prefetch ring, and in the register
    form, with several CTA shapes
    (consumer warps, ring stages, rows per CTA; 0 = automatic), 2D and 3D,
    against the numpy oracle: bit-identical."""
    from starmap_b200 import _lib
    from starmap_b200.solver import setup_gpu
    staged, slices, stages, rows = shape
    par = starmap_init(cases.ALL[name]())
    nsteps = 7
    ref = O.starmap_solver(par, max_steps=nsteps)
    S, fs, solver, T = setup_gpu(par)
    try:
        solver.tune(_lib.SMG_TUNE_JIT_STAGED, staged)
        solver.tune(_lib.SMG_TUNE_JIT_SLICES, slices)
        solver.tune(_lib.SMG_TUNE_JIT_STAGES, stages)
        solver.tune(_lib.SMG_TUNE_JIT_ROWS, rows)
        solver.set_variant(_lib.SMG_VARIANT_JIT)
        solver.set_state(S.U0)
        solver.set_dt(fs["dt"])
        solver.run(nsteps)
        solver.sync()
        U = solver.get_state()
        v, form = solver.active_variant()
    finally:
        solver.close()
    assert v == _lib.SMG_VARIANT_JIT and form == ["register", "bulk-staged", "async-staged", "prefetch-ring"][staged], \
        (v, form)
    worst, mism = 0.0, 0
    for j in range(S.n_sys):
        worst = max(worst, rel_l2(U[j], ref.U[j]))
        mism += int(np.count_nonzero(U[j] != ref.U[j]))
    assert worst <= REL_L2_TOL, f"{name} {shape}: worst relative L2 {worst:.3e}"
    assert mism == 0, f"{name} {shape}: {mism} values differ"


@pytest.mark.parametrize("prefetch", [2, 3])
@pytest.mark.parametrize("name", ["lattice_p5_substep", "odd_mixed_bc", "pt3d_p3"])
def test_bulk_l2_prefetch_vs_oracle(name, prefetch):
    """SMG_TUNE_JIT_PREFETCH 2/3 (bulk L2 prefetches of a later group's rows)
    moves no data the kernels compute with: results stay bit-identical."""
    from starmap_b200 import _lib
    from starmap_b200.solver import setup_gpu
    par = starmap_init(cases.ALL[name]())
    ref = O.starmap_solver(par, max_steps=6)
    S, fs, solver, T = setup_gpu(par)
    try:
        solver.tune(_lib.SMG_TUNE_JIT_PREFETCH, prefetch)
        solver.set_variant(_lib.SMG_VARIANT_JIT)
        solver.set_state(S.U0)
        solver.set_dt(fs["dt"])
        solver.run(6)
        U = solver.get_state()
    finally:
        solver.close()
    for j in range(S.n_sys):
        assert np.count_nonzero(U[j] != ref.U[j]) == 0, (name, j)

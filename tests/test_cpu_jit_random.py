"""The generated kernels compile for every problem structure: hypothesis
draws small problems (closure and order, odd and unequal sizes, per-axis
boundary conditions, field or scalar coefficients, filter position) and the
generated source -- plain, family (batched) and adjoint forms -- must compile
with NVRTC for sm_100a (no GPU needed).  Descriptors the generator cannot
serve (state beyond 32-bit offsets, grid types inconsistent with the
couplings) are refused on the host."""
import pytest
from hypothesis import HealthCheck, given, settings

from starmap_b200 import _lib, starmap_init
from starmap_b200.batch import _tables
from starmap_b200.solver import first_step, handle_tables, jit_source, prepare
from test_cpu_jit import _nvrtc_available
from test_cpu_oracle_random import problems


@settings(max_examples=8, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(problems())
def test_generated_kernels_compile_for_random_problems(prob):
    if not _nvrtc_available():
        pytest.skip("NVRTC library not present")
    S = prepare(starmap_init(prob))
    fs = first_step(S)
    T = _tables(S, fs)
    src = jit_source(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, T.fields, **handle_tables(S, T), compile=3,
                     tune={_lib.SMG_TUNE_JIT_GROUP: 4, _lib.SMG_TUNE_JIT_SPLIT: 3})
    # every component is updated once per phase in the plain kernels
    plain = src.split("// ---- program (smg_fam_")[0]
    assert plain.count("double* Uj = U + pt + ") == S.n_sys


@settings(max_examples=6, deadline=None, derandomize=True, suppress_health_check=[HealthCheck.too_slow])
@given(problems())
def test_generated_adjoint_kernels_compile_for_random_problems(prob):
    """The adjoint's recording and backward-phase kernels (filters '' and
    'substep', the adjoint's scope) compile for drawn structures too."""
    if not _nvrtc_available():
        pytest.skip("NVRTC library not present")
    if prob.get("f_position", "") == "full":
        prob = dict(prob)
        prob.pop("f_position")
        prob.pop("filterfunction")
    S = prepare(starmap_init(prob))
    fs = first_step(S)
    T = _tables(S, fs)
    src = jit_source(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, T.fields, **handle_tables(S, T), compile=2,
                     tune={_lib.SMG_TUNE_JIT_GROUP: 4, _lib.SMG_TUNE_JIT_SPLIT: 3})
    assert "smg_adj_p1_0(" in src and "smg_adj_s1_0(" in src


def test_generator_refuses_state_beyond_32bit_offsets():
    """A 2D P7 problem on 7800 x 7800 cells holds 36 slots of about 61e6
    points, over 2^31 doubles in all: the generated kernels address
    components through 32-bit element offsets, so the generator refuses it
    on the host instead of reading wrapped offsets."""
    from starmap_b200 import configs
    S = prepare(starmap_init(configs.linesource(n=20, n_mom=7, tfinal=0.1)))
    T = _tables(S, first_step(S))
    assert all(getattr(v, "ndim", 0) == 0 for v, _ in T.fields)
    big = [1, 7800, 7800]
    with pytest.raises(_lib.SmgError, match="32-bit element offsets"):
        jit_source(big, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, T.fields, **handle_tables(S, T))


def test_create_refuses_grid_types_inconsistent_with_the_couplings():
    """With periodic boundaries every grid has the same extents, so only the
    grid types show a wrong gt: a component moved to another grid is refused."""
    import numpy as np
    from starmap_b200 import configs
    S = prepare(starmap_init(configs.linesource(n=20, n_mom=3, tfinal=0.1)))
    T = _tables(S, first_step(S))
    gt = np.array(S.gt, dtype=np.int32).reshape(S.n_sys, 3).copy()
    gt[1, 2] = 3 - gt[1, 2]
    with pytest.raises(_lib.SmgError, match="differ in axis"):
        jit_source(S.n, S.bc, S.h, gt, S.Mx, S.My, S.Mz, T.fields, **handle_tables(S, T))

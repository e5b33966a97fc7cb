"""Generated kernels (SMG_VARIANT_JIT): the source for every parity case is
produced from the host tables alone and compiles with NVRTC for sm_100a
(no GPU needed)."""
import numpy as np
import pytest

import cases
from starmap_b200 import _lib, starmap_init
from starmap_b200.batch import _tables
from starmap_b200.solver import first_step, handle_tables, jit_source, prepare


def _source(name, compile=False, block=64, group=8):
    S = prepare(starmap_init(cases.ALL[name]()))
    fs = first_step(S)
    T = _tables(S, fs)
    return S, jit_source(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, T.fields, **handle_tables(S, T),
                         block=block, group=group, compile=compile)


def _nvrtc_available():
    try:
        _source("one_d_p5", compile=True)
        return True
    except _lib.SmgError as e:
        if "not found" in str(e):
            return False
        raise


@pytest.mark.parametrize("name", sorted(cases.ALL))
def test_generated_source_structure(name):
    S, src = _source(name)
    n_a = sum(1 for j in range(S.n_sys) if int(np.sum(np.asarray(S.gt[j]) == 2)) % 2 == 1)
    assert "smg_jit_p1(" in src
    assert ("smg_jit_p0(" in src) == (n_a > 0)
    # one block per destination: every component is updated once per phase
    assert src.count("double* Uj = U + pt + ") == S.n_sys
    # one device function per group of 8 destinations, called from the dispatch kernels
    ngroups = (n_a + 7) // 8 + (S.n_sys - n_a + 7) // 8
    assert src.count("__noinline__ void smg_g") == ngroups


@pytest.mark.parametrize("name", ["lin_p7_periodic", "odd_mixed_bc", "pt3d_p3", "lattice_p4_full", "spn_3d"])
def test_generated_source_compiles(name):
    if not _nvrtc_available():
        pytest.skip("NVRTC library not present")
    _source(name, compile=True, block=128, group=3)


def test_bad_tuning_rejected():
    with pytest.raises(_lib.SmgError):
        _source("one_d_p5", block=48)

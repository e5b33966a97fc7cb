"""The roofline numerator: algorithmic HBM bytes per step of the fused-phase
design.  Each phase reads every component once and writes its destinations
once, plus one read of each distinct coefficient array it uses; a step is
phase A, phase B, phase A (starmap_solver.m:310), or, with the two phase-A
passes of neighbouring steps fused, one A pass and one B pass."""
import numpy as np
import pytest

from starmap_b200 import configs, starmap_init
from starmap_b200.batch import _tables
from starmap_b200.roofline import algorithmic_bytes_per_step
from starmap_b200.solver import first_step, prepare


def _setup(prob):
    S = prepare(starmap_init(prob))
    return S, _tables(S, first_step(S))


def test_linesource_p7_bytes_per_update():
    """36 components (20 in phase A, 16 in phase B), all on n x n grids with
    periodic boundaries and scalar coefficients: 8 (3*36 + 2*20 + 16) / 36
    = 36.44 B per update unfused, 24 B fused."""
    n = 40
    S, T = _setup(configs.linesource(n=n, n_mom=7, tfinal=0.1))
    cells = n * n
    plain = algorithmic_bytes_per_step(S, T)
    fused = algorithmic_bytes_per_step(S, T, fused=True)
    assert (plain["n_outer"], plain["n_inner"]) == (20, 16)
    assert plain["step"] == 8 * cells * (3 * 36 + 2 * 20 + 16)
    assert plain["step"] / (36 * cells) == pytest.approx(36.444, abs=1e-3)
    assert fused["step"] == 24 * 36 * cells
    assert plain["state_bytes"] == fused["state_bytes"] == 8 * 36 * cells


@pytest.mark.parametrize("f_position", ["substep", "full"])
def test_lattice_bytes_split_into_state_and_coefficients(f_position):
    """Closed boundaries add a face row and column to staggered grids; the
    state part follows the per-component point counts and the coefficient
    part is one read per distinct array field a phase uses."""
    n = 14
    S, T = _setup(configs.lattice(n=n, n_mom=5, tfinal=0.1, f_position=f_position))
    pts = [int(np.prod([n + 1 if (g == 2 and S.bc[d] == 1) else n for d, g in enumerate(S.G(j))][1:]))
           for j in range(S.n_sys)]
    outer = [j for j in range(S.n_sys) if sum(g == 2 for g in S.G(j)) % 2 == 1]
    inner = [j for j in range(S.n_sys) if j not in outer]
    r = algorithmic_bytes_per_step(S, T)
    state = 8 * (3 * sum(pts) + 2 * sum(pts[j] for j in outer) + sum(pts[j] for j in inner))
    coef = r["step"] - state - r["full_filter"]
    n_arrays = sum(np.ndim(v) > 0 for v, _ in T.fields)
    assert n_arrays > 0
    assert 3 * 8 * n * n <= coef <= 3 * 8 * (n + 1) ** 2 * n_arrays   # every phase reads an array sigma
    if f_position == "full":
        assert r["full_filter"] >= 2 * 8 * sum(pts[1:])
    else:
        assert r["full_filter"] == 0

"""CPU-only tests: library exports, closures, classification, host logic."""
import ctypes
import os
import re

import numpy as np
import pytest

from oracle import solver_np as O
from starmap_b200 import _lib, closure_pn, closure_spn, starmap_init
from starmap_b200.init import capargs, hook, nargin
from starmap_b200.solver import colon, expm1div, step_times

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def header_symbols():
    txt = open(os.path.join(ROOT, "include", "starmap_gpu.h")).read()
    return sorted(set(re.findall(r"\b(smg_[a-z_]+)\s*\(", txt)))


def test_library_loads_and_exports_every_header_symbol():
    L = ctypes.CDLL(_lib.LIB_PATH)
    syms = header_symbols()
    assert len(syms) >= 15
    for s in syms:
        assert hasattr(L, s), f"{s} declared in include/starmap_gpu.h but not exported"
    assert set(syms) <= set(_lib.SIGNATURES), "ctypes binding lacks a header symbol"
    assert _lib.lib().smg_version().decode().startswith("starmap_b200")
    assert _lib.lib().smg_device_count() >= 0


def test_ctypes_signatures_match_header_prototypes():
    """Every prototype of include/starmap_gpu.h has a ctypes binding with the
    same number of parameters, pointer parameters bound as pointers, and
    void returns as None."""
    txt = re.sub(r"/\*.*?\*/", "", open(os.path.join(ROOT, "include", "starmap_gpu.h")).read(), flags=re.S)
    protos = re.findall(r"^\s*((?:const\s+)?\w+\s*\**)\s*(smg_\w+)\s*\(([^;{]*?)\)\s*;", txt, flags=re.M)
    assert {p[1] for p in protos} == set(_lib.SIGNATURES)
    for ret, name, args in protos:
        restype, argtypes = _lib.SIGNATURES[name]
        assert (ret.strip() == "void") == (restype is None), name
        params = [] if args.strip() in ("", "void") else args.split(",")
        assert len(params) == len(argtypes), name
        for param, ct in zip(params, argtypes):
            is_ptr = "*" in param or "[" in param
            ct_ptr = ct in (ctypes.c_void_p, ctypes.c_char_p) or issubclass(ct, ctypes._Pointer)
            assert is_ptr == ct_ptr, (name, param)


def test_ctypes_struct_layouts_match_the_c_compiler():
    """smg_field and smg_problem: size and every member offset of the ctypes
    mirror agree with the C compiler's layout of the header (static
    assertions checked by gcc -fsyntax-only; nothing is written)."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not present")
    lines = ["#include <stddef.h>", '#include "starmap_gpu.h"']
    for st in (_lib.smg_field, _lib.smg_problem):
        name = st.__name__
        lines.append(f'_Static_assert(sizeof({name}) == {ctypes.sizeof(st)}, "sizeof {name}");')
        for fname, _ in st._fields_:
            off = getattr(st, fname).offset
            lines.append(f'_Static_assert(offsetof({name}, {fname}) == {off}, "{name}.{fname}");')
    r = subprocess.run([gcc, "-fsyntax-only", "-x", "c", "-I", os.path.join(ROOT, "include"), "-"],
                       input="\n".join(lines) + "\n", capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


@pytest.mark.parametrize("lang,std", [("c", "c99"), ("c++", "c++11")])
def test_header_compiles_standalone(lang, std):
    """A MEX gateway in plain C or any C++ host includes the header alone."""
    import shutil
    import subprocess
    cc = shutil.which("gcc" if lang == "c" else "g++")
    if cc is None:
        pytest.skip("compiler not present")
    r = subprocess.run([cc, f"-std={std}", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only", "-x", lang,
                        "-I", os.path.join(ROOT, "include"), "-"],
                       input='#include "starmap_gpu.h"\n', capture_output=True, text=True)
    assert r.returncode == 0, r.stderr


def test_create_rejects_bad_descriptor():
    L = _lib.lib()
    p = _lib.smg_problem()
    p.n_sys = 0
    h = ctypes.c_void_p()
    assert L.smg_create(ctypes.byref(p), ctypes.byref(h)) == _lib.SMG_EINVAL
    assert b"n_sys" in L.smg_last_error(None)
    assert L.smg_create(None, ctypes.byref(h)) == _lib.SMG_EINVAL


@pytest.mark.parametrize("n,msg", [((1, 65536, 32768), b"2^31"), ((1, 1, (1 << 30) + 1), b"n[d]")])
def test_create_refuses_grids_beyond_32bit_point_index(n, msg):
    """A component whose padded slot holds 2^31 points or more is refused
    before any device work (the kernels index a point with 32 bits)."""
    L = _lib.lib()
    p = _lib.smg_problem()
    p.n_sys = 1
    p.n[:] = n
    p.bc[:] = (0, 0, 0)
    p.h[:] = (1.0, 1e-3, 1e-3)
    gt = (ctypes.c_int32 * 3)(1, 1, 1)
    M = (ctypes.c_double * 1)(0.0)
    tab = (ctypes.c_int32 * 1)(-1)
    f = (_lib.smg_field * 1)()
    f[0].scalar = 1.0
    f[0].grid[:] = (1, 1, 1)
    p.gt, p.Mx, p.My, p.Mz = gt, M, M, M
    p.n_fields, p.fields = 1, f
    p.sigma_t, p.source = tab, tab
    p.sigma_a, p.decay_a, p.filter_mode = 0, -1, 0
    h = ctypes.c_void_p()
    assert L.smg_create(ctypes.byref(p), ctypes.byref(h)) == _lib.SMG_EINVAL
    assert msg in L.smg_last_error(None)
    assert not h.value


@pytest.mark.parametrize("N,lam", [(7, 0.960290), (39, 0.998238), (15, 0.989401)])
def test_pn2d_eigenvalue_pins(N, lam):
    # largest |eigenvalue| of Mz equals the largest root of the Legendre
    # polynomial P_{N+1}: an independent known answer for the closure tables
    _, _, _, Mz = closure_pn(N, 2)
    roots = np.polynomial.legendre.leggauss(N + 1)[0]
    ev = np.max(np.abs(np.linalg.eigvalsh(Mz)))
    assert abs(ev - roots.max()) < 1e-12
    assert abs(ev - lam) < 5e-7


def test_pn3d_tables():
    o, Mx, My, Mz = closure_pn(9, 3)
    assert Mz.shape == (100, 100)
    for M in (Mx, My, Mz):
        np.testing.assert_array_equal(M, M.T)
    np.testing.assert_array_equal(o, np.ceil(np.sqrt(np.arange(1, 101)) - 1))
    roots = np.polynomial.legendre.leggauss(10)[0]
    assert abs(np.max(np.abs(np.linalg.eigvalsh(Mz))) - roots.max()) < 1e-12


@pytest.mark.parametrize("cl,N,dim", [("P", 1, 2), ("P", 7, 2), ("P", 39, 2), ("P", 2, 3), ("P", 9, 3),
                                      ("SP", 5, 2), ("SP", 9, 3), ("P", 5, 1), ("SP", 4, 2)])
def test_native_classification_matches_oracle(cl, N, dim):
    f = closure_pn if cl == "P" else closure_spn
    _, Mx, My, Mz = f(N, dim)
    gt = _lib.classify(Mx, My, Mz)
    _, _, _, _, gx, gy, gz = O._classify(Mx, My, Mz)
    np.testing.assert_array_equal(gt, np.stack([gx, gy, gz], 1))


def test_classification_refuses_unstaggerable_couplings():
    """Component 3 reached from component 1 along y (grid 1,2) and, through
    component 2, along x twice (grid 1,1): no staggered grid types exist, and
    the classification says so instead of picking one."""
    Mx = np.array([[0., 1, 0], [1, 0, 1], [0, 1, 0]])
    My = np.array([[0., 0, 1], [0, 0, 0], [1, 0, 0]])
    Mz = np.zeros((3, 3))
    with pytest.raises(_lib.SmgError, match="admit no staggered grid types"):
        _lib.classify(Mx, My, Mz)
    with pytest.raises(_lib.SmgError, match="not connected"):
        _lib.classify(np.zeros((2, 2)), np.zeros((2, 2)), np.zeros((2, 2)))


def test_phase_partition_counts():
    # component sets of the benchmark configurations
    def counts(N, dim):
        _, Mx, My, Mz = closure_pn(N, dim)
        gt = _lib.classify(Mx, My, Mz)
        outer = int(np.sum((gt == 2).sum(1) % 2 == 1))
        return Mz.shape[0], outer, Mz.shape[0] - outer
    assert counts(7, 2) == (36, 20, 16)
    assert counts(39, 2) == (820, 420, 400)
    assert counts(9, 3) == (100, 55, 45)
    assert counts(15, 2) == (136, 72, 64)


def test_expm1div_branch():
    x = np.array([-1e-5, 1e-4, -2e-4, 2.0000001e-4, -3e-4, -1.0, 0.0])
    y = expm1div(x)
    for xi, yi in zip(x, y):
        if abs(xi) > 2e-4:
            assert yi == (np.exp(xi) - 1) / xi
        else:
            assert yi == 1 + xi * .5 + xi ** 2 / 6
    assert expm1div(0.0) == 1.0


def test_colon_and_step_count():
    v = colon(0.015, 0.03, 3.0 - 0.015)
    assert len(v) == 100 and v[0] == 0.015
    ts = step_times(0.015, 1.0)
    assert len(ts) == 67 and ts[-1] >= 1.0       # overshoots tfinal
    assert len(step_times(0.01, 3.2)) in (320, 321)


def test_nargin_semantics():
    assert nargin(lambda x, y: 0) == 2
    assert nargin(lambda *a: 0) == -1
    assert nargin(hook(lambda *a: 0, 4)) == 4
    assert capargs(lambda x: x, 1, 2, 3) == 1


def test_init_wraps_2d_hooks_and_defaults():
    par = starmap_init(dict(closure="P", n_mom=3, ax=[0, 1, 0, 2], n=[4, 5], bc=[1, 0],
                            ic=lambda x, y: x + 10 * y, source=lambda x, y, t: t))
    assert par["dim"] == 2 and par["n"] == [1, 4, 5] and par["bc"] == [1, 1, 0]
    assert par["ax"] == [0, 1, 0, 1, 0, 2]
    assert nargin(par["ic"]) == 3 and par["ic"](None, 2.0, 3.0) == 32.0
    assert nargin(par["source"]) == 4
    assert list(par["source_ind"]) == [1]
    assert par["tfinal"] == 1.0 and par["cn"] == 0.99
    with pytest.raises(ValueError):
        starmap_init(dict(closure="P", n_mom=3, ax=[0, 1, 0, 2], n=[4]))
    with pytest.raises(ValueError):
        starmap_init(dict(closure="P", n_mom=3, ax=[0, 1, 0, 1], ic=lambda x: x))


@pytest.mark.parametrize("prob", [
    dict(closure="P", n_mom=3),                                            # none of ax, n, bc
    dict(closure="P", n_mom=3, ax=[0, 1, 0, 1], bc=[1, 1, 1]),             # ax and bc disagree
    dict(closure="P", n_mom=3, n=[4, 4], bc=[0, 0, 0]),                    # n and bc disagree
    dict(closure="P", n_mom=3, ax=[0, 1, 0, 1], n=[4, 4], sigma_a=lambda a, b, c, d, e: a),   # hook arity
    dict(closure="P", n_mom=3, ax=[0, 1, 0, 1], n=[4, 4], source=lambda: 1.0),                # hook arity
])
def test_init_rejects_inconsistent_problems(prob):
    """starmap_init.m:36-60 and the hook-arity checks: inconsistent ax/n/bc
    and hooks of an unsupported number of arguments are errors."""
    with pytest.raises(ValueError):
        starmap_init(prob)


def test_batch_refuses_full_filter_before_device_work():
    """The batched solver does not apply the full-step filter, so an instance
    with f_position 'full' is refused at creation (before any device work)."""
    from starmap_b200 import _lib, configs
    from starmap_b200.batch import setup_batch
    probs = configs.batched_sweep(n_inst=2, seed=5, edges=(16,), orders=(1,))
    probs[1].update(filterfunction=configs.exp_filter(2, 2.0), f_position="full")
    with pytest.raises(_lib.SmgError, match="full"):
        setup_batch([starmap_init(p) for p in probs])


def test_batch_refuses_time_dependent_problems():
    """A batch keeps each instance's first-step coefficients and dt, so
    time-dependent hooks are refused at set-up (on the host)."""
    import cases
    from starmap_b200 import configs
    from starmap_b200.batch import setup_batch
    good = starmap_init(configs.batched_sweep(n_inst=1, seed=5, edges=(16,), orders=(1,))[0])
    for bad in (cases.td_sigma(), cases.boxes_td_source()):
        with pytest.raises(ValueError, match="time-dependent"):
            setup_batch([good, starmap_init(bad)])



def test_mex_gateway_compiles_strictly_against_the_header():
    """matlab/starmap_solver_mex.c is C99 against include/starmap_gpu.h and the
    test-only stand-in of the MATLAB C API (tests/mex/mex.h): no warnings with
    -Wall -Wextra -pedantic."""
    import shutil
    import subprocess
    gcc = shutil.which("gcc")
    if gcc is None:
        pytest.skip("gcc not present")
    r = subprocess.run([gcc, "-std=c99", "-Wall", "-Wextra", "-pedantic", "-Werror", "-fsyntax-only",
                        "-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "tests", "mex"),
                        os.path.join(ROOT, "matlab", "starmap_solver_mex.c")], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr

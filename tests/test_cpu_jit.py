"""Generated kernels (SMG_VARIANT_JIT): the source for every parity case is
produced from the host tables alone and compiles with NVRTC for sm_100a
(no GPU needed)."""
import numpy as np
import pytest

import cases
from starmap_b200 import _lib, starmap_init
from starmap_b200.batch import _tables
from starmap_b200.solver import first_step, handle_tables, jit_source, prepare


def _source(name, compile=False, block=64, group=8, **tune):
    S = prepare(starmap_init(cases.ALL[name]()))
    fs = first_step(S)
    T = _tables(S, fs)
    settings = {_lib.SMG_TUNE_JIT_BLOCK: block, _lib.SMG_TUNE_JIT_GROUP: group}
    settings.update({getattr(_lib, "SMG_TUNE_JIT_" + k.upper()): v for k, v in tune.items()})
    return S, jit_source(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, T.fields, **handle_tables(S, T),
                         compile=compile, tune=settings)


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
    S, src = _source(name, split=4, calls=0, staged=0)
    n_a = sum(1 for j in range(S.n_sys) if int(np.sum(np.asarray(S.gt[j]) == 2)) % 2 == 1)
    assert "smg_jit_p1_0(" in src
    assert ("smg_jit_p0_0(" in src) == (n_a > 0)
    # one block per destination: every component is updated once per phase
    assert src.count("double* Uj = U + pt + ") == S.n_sys
    # groups of at most 8 destinations of one grid type (one function each), 4 groups per kernel
    import re
    ga = len(set(re.findall(r"void (smg_g0_\d+)\(", src)))
    gb = len(set(re.findall(r"void (smg_g1_\d+)\(", src)))
    assert (n_a + 7) // 8 <= ga <= n_a and (S.n_sys - n_a + 7) // 8 <= gb <= S.n_sys - n_a
    assert src.count("__global__") == (ga + 3) // 4 + (gb + 3) // 4


@pytest.mark.parametrize("loader", [1, 2])
@pytest.mark.parametrize("name", sorted(cases.ALL))
def test_staged_source_structure(name, loader):
    """The staged forms: one function per group, one block per destination;
    with bulk copies every copy is counted in the bytes the stage expects,
    with asynchronous copies every staged row segment is copied once per row
    and every x source's two halos once."""
    import re
    S, src = _source(name, split=4, calls=0, staged=loader, slices=3)
    n_a = sum(1 for j in range(S.n_sys) if int(np.sum(np.asarray(S.gt[j]) == 2)) % 2 == 1)
    assert src.count("double* Uj = U + pt + ") == S.n_sys
    ga = len(set(re.findall(r"void (smg_s0_\d+)\(", src)))
    gb = len(set(re.findall(r"void (smg_s1_\d+)\(", src)))
    assert (n_a + 7) // 8 <= ga <= n_a and (S.n_sys - n_a + 7) // 8 <= gb <= S.n_sys - n_a
    assert src.count("__global__") == (ga + 3) // 4 + (gb + 3) // 4
    assert "multicast" not in src
    for body in src.split("static __device__ __forceinline__ void smg_s")[1:]:
        body = body.split("\n}\n")[0]
        if loader == 1:
            # the expected bytes name as many copies as the producer issues
            m = re.search(r"const unsigned tx = (\d+)u \* xb \+ (\d+)u \* db;", body)
            assert m, body[:200]
            assert body.count("bulk_ld(stg") == int(m.group(1)) + int(m.group(2))
            assert body.count(", xb, &bar[s]);") == int(m.group(1))
        else:
            assert "bulk_ld(" not in body and "mb_wait(" not in body
            slots = set(int(v) for v in re.findall(r"cpa\(stg \+ (\d+) \+ 2 \* lane", body))
            assert len(slots) == body.count("cpa(stg + ")           # each slot copied once
            assert sorted(slots) == [68 * i + 2 for i in range(len(slots))]   # slots 0..n-1
            assert body.count("cpa(hd + ") == len(set(re.findall(r"double X(\d+)_a0", body))) or \
                body.count("cpa(hd + ") >= 1 or "X" not in body


@pytest.mark.parametrize("name", ["lin_p7_periodic", "odd_mixed_bc", "pt3d_p3", "lattice_p4_full", "spn_3d"])
@pytest.mark.parametrize("layout", [dict(calls=0, split=4, xpair=0), dict(calls=1, split=2, xpair=1),
                                    dict(calls=0, split=16, staged=0),
                                    dict(calls=0, split=4, staged=1, slices=3, stages=2, rows=7),
                                    dict(calls=0, split=4, staged=2, slices=5, stages=4, rows=3),
                                    dict(calls=0, split=0, xpair=1), dict(calls=0, split=16, prefetch=1),
                                    dict(calls=0, split=16, xpair=2), dict(calls=0, split=16, band=5),
                                    dict(calls=0, split=16, const=1)])
def test_generated_source_compiles(name, layout):
    if not _nvrtc_available():
        pytest.skip("NVRTC library not present")
    _source(name, compile=True, block=128, group=3, **layout)


def test_bad_tuning_rejected():
    with pytest.raises(_lib.SmgError):
        _source("one_d_p5", block=48)
    for lanes in (-1, 65):
        with pytest.raises(_lib.SmgError):
            _source("one_d_p5", lanes=lanes)
    _source("one_d_p5", lanes=2)   # launch setting: the source is the same
    assert _source("one_d_p5", lanes=2)[1] == _source("one_d_p5")[1]


@pytest.mark.parametrize("name", ["odd_mixed_bc", "pt3d_p3", "lattice_p5_substep", "lattice_p6_nofilter"])
def test_adjoint_kernels_compile(name):
    if not _nvrtc_available():
        pytest.skip("NVRTC library not present")
    S, src = _source(name, compile=2, block=64, group=3)
    assert "smg_adj_p0_0(" in src and "smg_adj_p1_0(" in src and "_r(" in src


@pytest.mark.parametrize("name", ["odd_mixed_bc", "pt3d_p3", "lattice_p5_substep", "spn_3d", "aniso_2d"])
def test_family_kernels_compile(name):
    """The batched solver's family kernels (shared-load groups with the grid
    taken from the instance's geometry at run time) compile for sm_100a."""
    if not _nvrtc_available():
        pytest.skip("NVRTC library not present")
    S, src = _source(name, compile=3, block=64, group=4)
    assert "smg_fam_p1_0(" in src and "const FamGeom& G" in src
    # one block per destination in the family kernels too
    fam = src[src.index("// ---- program (smg_fam_"):]
    assert fam.count("double* Uj = U + pt + ") == S.n_sys


@pytest.mark.parametrize("split", [1, 16])
@pytest.mark.parametrize("name", ["lattice_p5_substep", "pt3d_p3", "spn_3d"])
def test_generated_source_is_deterministic(name, split):
    """The per-process compile cache is keyed by source text, so the
    generator gives the same text for the same problem, also after another
    problem was generated in between; with one group per program the
    programs are written on several threads and must keep their order."""
    _, a = _source(name, split=split)
    _source("odd_mixed_bc", split=4)
    _, b = _source(name, split=split)
    assert a == b
    names = [l.split("(")[1].rstrip(")") for l in a.splitlines() if l.startswith("// ---- program")]
    assert len(names) >= 2
    for phase in ("p0", "p1"):
        firsts = [int(n.split("_")[-1]) for n in names if n.startswith("smg_jit_" + phase + "_")]
        assert firsts == sorted(firsts) and len(firsts) == len(set(firsts))


_CACHE_PROBE = r"""
import ctypes, json, sys
sys.path.insert(0, {root!r}); sys.path.insert(0, {tests!r})
from test_cpu_jit import _source
from starmap_b200 import _lib
_source("lattice_p5_substep", compile=True, split=2)
c, d = ctypes.c_int64(), ctypes.c_int64()
_lib.lib().smg_jit_stats(ctypes.byref(c), ctypes.byref(d))
print(json.dumps([c.value, d.value]))
"""


def test_compiled_kernels_are_cached_on_disk_across_processes():
    """A second process generating the same problem's kernels loads them from
    the on-disk cache instead of compiling (smg_jit_stats); a damaged cache
    file is not used; SMG_JIT_CACHE=0 compiles again and writes nothing."""
    import json
    import os
    import shutil
    import subprocess
    import sys
    if not _nvrtc_available():
        pytest.skip("NVRTC library not present")
    here = os.path.dirname(os.path.abspath(__file__))
    root = os.path.dirname(here)
    d = os.path.join(root, "_build", "cache_test_%d" % os.getpid())
    shutil.rmtree(d, ignore_errors=True)
    code = _CACHE_PROBE.format(root=root, tests=here)

    def run(**env):
        e = dict(os.environ, SMG_JIT_CACHE_DIR=d, **env)
        out = subprocess.run([sys.executable, "-c", code], env=e, capture_output=True, text=True, timeout=600)
        assert out.returncode == 0, out.stderr[-2000:]
        return json.loads(out.stdout.strip().splitlines()[-1])

    try:
        compiled, from_disk = run()
        assert compiled > 0 and from_disk == 0
        assert len([f for f in os.listdir(d) if f.endswith(".cubins")]) == 1
        compiled, from_disk = run()
        assert compiled == 0 and from_disk > 0
        # a damaged file (one cubin byte flipped, or cut short) is ignored,
        # compiled again and rewritten
        f = os.path.join(d, [f for f in os.listdir(d) if f.endswith(".cubins")][0])
        good = open(f, "rb").read()
        assert good.startswith(b"SMGCUB2\n")
        bad = bytearray(good)
        bad[-100] ^= 0x40
        for damaged in (bytes(bad), good[:-9]):
            open(f, "wb").write(damaged)
            compiled, from_disk = run()
            assert compiled > 0 and from_disk == 0
            assert open(f, "rb").read() == good
        shutil.rmtree(d)
        compiled, from_disk = run(SMG_JIT_CACHE="0")
        assert compiled > 0 and from_disk == 0 and not os.path.exists(d)
    finally:
        shutil.rmtree(d, ignore_errors=True)

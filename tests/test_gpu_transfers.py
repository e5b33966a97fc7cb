"""State transfers: page-locked host arrays are moved by one kernel that
reads or writes them in place (unified addressing), pageable ones through the
device staging buffer; both forms give the same state bit for bit, for
uploads, downloads and the output-time interpolation."""
import numpy as np
import pytest

import cases
from starmap_b200 import _lib, starmap_init
from starmap_b200.solver import setup_gpu

pytestmark = pytest.mark.gpu


def pinned_like(arrs):
    torch = pytest.importorskip("torch")
    out = []
    for a in arrs:
        b = torch.empty(a.size, dtype=torch.float64, pin_memory=True).numpy()
        b[:] = np.asarray(a, dtype=np.float64).ravel(order="F")
        out.append(b.reshape(a.shape, order="F"))
    return out


def pinned_block(arrs):
    """Page-locked arrays carved in order from one block (host-adjacent)."""
    torch = pytest.importorskip("torch")
    block = torch.empty(sum(a.size for a in arrs), dtype=torch.float64, pin_memory=True).numpy()
    out, o = [], 0
    for a in arrs:
        v = block[o:o + a.size]
        v[:] = np.asarray(a, dtype=np.float64).ravel(order="F")
        out.append(v.reshape(a.shape, order="F"))
        o += a.size
    return out


@pytest.mark.parametrize("name", ["lattice_p5_substep", "odd_mixed_bc", "box3d_bc1_p2_full"])
def test_block_carved_arrays_transfer_exactly(name):
    """Page-locked arrays carved from one block take the staged path with
    merged copies; values arrive intact both ways, also for the output-time
    interpolation, and equal those of separate arrays."""
    par = starmap_init(cases.ALL[name]())
    res = []
    for carve in (pinned_block, pinned_like):
        S, fs, solver, T = setup_gpu(par)
        try:
            rng = np.random.default_rng(4)
            U0 = [rng.standard_normal(solver.extents(j)) for j in range(S.n_sys)]
            solver.set_state(carve(U0))
            outs = dict(enumerate(carve([np.zeros(solver.extents(j)) for j in range(S.n_sys)])))
            back = solver.get_state(out={j: o.reshape(-1, order="F") for j, o in outs.items()})
            for j in range(S.n_sys):
                np.testing.assert_array_equal(back[j], U0[j])
            solver.set_dt(fs["dt"])
            solver.run(2)
            solver.snapshot()
            solver.run(1)
            outs = dict(enumerate(carve([np.zeros(solver.extents(j)) for j in range(S.n_sys)])))
            V = solver.get_interp(0.3, out={j: o.reshape(-1, order="F") for j, o in outs.items()})
            res.append({j: np.array(V[j]) for j in V})
        finally:
            solver.close()
    for j in res[0]:
        np.testing.assert_array_equal(res[0][j], res[1][j])


@pytest.mark.parametrize("name", ["lattice_p5_substep", "odd_mixed_bc", "box3d_bc1_p2_full"])
def test_direct_and_staged_transfers_agree(name):
    par = starmap_init(cases.ALL[name]())
    res = {}
    for direct in (1, 0):
        S, fs, solver, T = setup_gpu(par)
        try:
            solver.tune(_lib.SMG_TUNE_DIRECT_XFER, direct)
            rng = np.random.default_rng(3)
            U0 = [rng.standard_normal(solver.extents(j)) for j in range(S.n_sys)]
            solver.set_state(pinned_like(U0) if direct else U0)
            back = solver.get_state(out={j: pinned_like([np.zeros(solver.extents(j))])[0] for j in range(S.n_sys)}
                                    if direct else None)
            for j in range(S.n_sys):
                np.testing.assert_array_equal(back[j], U0[j])
            solver.set_dt(fs["dt"])
            solver.run(2)
            solver.snapshot()
            solver.run(1)
            outs = {j: pinned_like([np.zeros(solver.extents(j))])[0] for j in range(S.n_sys)} if direct else None
            U = solver.get_state(out=outs)
            outs2 = {j: pinned_like([np.zeros(solver.extents(j))])[0] for j in range(S.n_sys)} if direct else None
            V = solver.get_interp(0.3, out=outs2)
            res[direct] = ({j: np.array(U[j]) for j in U}, {j: np.array(V[j]) for j in V})
        finally:
            solver.close()
    for j in res[0][0]:
        np.testing.assert_array_equal(res[1][0][j], res[0][0][j])
        np.testing.assert_array_equal(res[1][1][j], res[0][1][j])


def _at_page(size, shift):
    """A float64 array of `size` values starting `shift` bytes after a page
    boundary (page-aligned arrays make a registration of the array's first
    pages include its first byte)."""
    raw = np.empty(size + 1024, dtype=np.float64)
    skip = ((-raw.ctypes.data) % 4096 + shift) // 8
    return raw[skip:skip + size]


@pytest.mark.parametrize("shift", [0, 8])
@pytest.mark.parametrize("half", ["first", "second"])
def test_partly_page_locked_arrays_take_the_staged_path(half, shift):
    """An array of which only one half is page-locked (cudaHostRegister of a
    sub-range) must not be read or written in place (its other half has no
    device mapping), nor be the range of one copy when its first byte is
    page-locked (the driver refuses a copy past the registration).  Such
    arrays go through a host bounce buffer or the staging buffer, and the
    values arrive intact in both directions."""
    torch = pytest.importorskip("torch")
    cudart = torch.cuda.cudart()
    from starmap_b200 import configs
    par = starmap_init(configs.lattice(n=100, n_mom=3))   # 80 KB per component
    S, fs, solver, T = setup_gpu(par)
    regs = []
    try:
        rng = np.random.default_rng(5)
        U0, outs = [], {}
        for j in range(S.n_sys):
            e = solver.extents(j)
            a = _at_page(int(np.prod(e)), shift).reshape(e, order="F")
            a[...] = rng.standard_normal(e)
            U0.append(a)
            outs[j] = _at_page(int(np.prod(e)), shift)
        page = 4096
        for a in list(U0) + list(outs.values()):
            nbytes = a.size * 8
            assert nbytes > 4 * page
            base = a.ctypes.data
            lo = (base + page - 1) // page * page           # whole pages inside the array
            hi = (base + nbytes) // page * page
            mid = (lo + hi) // 2 // page * page
            start, end = (lo, mid) if half == "first" else (mid, hi)
            assert int(cudart.cudaHostRegister(start, end - start, 0)) == 0
            regs.append(start)
        solver.set_state(U0)
        back = solver.get_state(out=outs)
        for j in range(S.n_sys):
            np.testing.assert_array_equal(back[j], U0[j])
    finally:
        for r in regs:
            cudart.cudaHostUnregister(r)
        solver.close()


def pinned_block(arrs):
    """Page-locked arrays carved in order from one block (host-adjacent)."""
    torch = pytest.importorskip("torch")
    block = torch.empty(sum(a.size for a in arrs), dtype=torch.float64, pin_memory=True).numpy()
    out, o = [], 0
    for a in arrs:
        v = block[o:o + a.size]
        v[:] = np.asarray(a, dtype=np.float64).ravel(order="F")
        out.append(v.reshape(a.shape, order="F"))
        o += a.size
    return out


@pytest.mark.parametrize("name", ["lattice_p5_substep", "odd_mixed_bc", "box3d_bc1_p2_full"])
def test_block_carved_arrays_transfer_exactly(name):
    """Page-locked arrays carved from one block take the staged path with
    merged copies; values arrive intact both ways, also for the output-time
    interpolation, and equal those of separate arrays."""
    par = starmap_init(cases.ALL[name]())
    res = []
    for carve in (pinned_block, pinned_like):
        S, fs, solver, T = setup_gpu(par)
        try:
            rng = np.random.default_rng(4)
            U0 = [rng.standard_normal(solver.extents(j)) for j in range(S.n_sys)]
            solver.set_state(carve(U0))
            outs = dict(enumerate(carve([np.zeros(solver.extents(j)) for j in range(S.n_sys)])))
            back = solver.get_state(out={j: o.reshape(-1, order="F") for j, o in outs.items()})
            for j in range(S.n_sys):
                np.testing.assert_array_equal(back[j], U0[j])
            solver.set_dt(fs["dt"])
            solver.run(2)
            solver.snapshot()
            solver.run(1)
            outs = dict(enumerate(carve([np.zeros(solver.extents(j)) for j in range(S.n_sys)])))
            V = solver.get_interp(0.3, out={j: o.reshape(-1, order="F") for j, o in outs.items()})
            res.append({j: np.array(V[j]) for j in V})
        finally:
            solver.close()
    for j in res[0]:
        np.testing.assert_array_equal(res[0][j], res[1][j])


@pytest.mark.parametrize("name", ["lattice_p5_substep", "odd_mixed_bc", "box3d_bc1_p2_full"])
def test_direct_and_staged_transfers_agree(name):
    par = starmap_init(cases.ALL[name]())
    res = {}
    for direct in (1, 0):
        S, fs, solver, T = setup_gpu(par)
        try:
            solver.tune(_lib.SMG_TUNE_DIRECT_XFER, direct)
            rng = np.random.default_rng(3)
            U0 = [rng.standard_normal(solver.extents(j)) for j in range(S.n_sys)]
            solver.set_state(pinned_like(U0) if direct else U0)
            back = solver.get_state(out={j: pinned_like([np.zeros(solver.extents(j))])[0] for j in range(S.n_sys)}
                                    if direct else None)
            for j in range(S.n_sys):
                np.testing.assert_array_equal(back[j], U0[j])
            solver.set_dt(fs["dt"])
            solver.run(2)
            solver.snapshot()
            solver.run(1)
            outs = {j: pinned_like([np.zeros(solver.extents(j))])[0] for j in range(S.n_sys)} if direct else None
            U = solver.get_state(out=outs)
            outs2 = {j: pinned_like([np.zeros(solver.extents(j))])[0] for j in range(S.n_sys)} if direct else None
            V = solver.get_interp(0.3, out=outs2)
            res[direct] = ({j: np.array(U[j]) for j in U}, {j: np.array(V[j]) for j in V})
        finally:
            solver.close()
    for j in res[0][0]:
        np.testing.assert_array_equal(res[1][0][j], res[0][0][j])
        np.testing.assert_array_equal(res[1][1][j], res[0][1][j])


@pytest.mark.parametrize("half", ["first", "second"])
def test_partly_page_locked_arrays_take_the_staged_path(half):
    """An array of which only one half is page-locked (cudaHostRegister of a
    sub-range) must not be read or written in place: its other half has no
    device mapping.  Such arrays go through the staging buffer and the values
    arrive intact in both directions."""
    torch = pytest.importorskip("torch")
    cudart = torch.cuda.cudart()
    from starmap_b200 import configs
    par = starmap_init(configs.lattice(n=100, n_mom=3))   # 80 KB per component
    S, fs, solver, T = setup_gpu(par)
    regs = []
    try:
        rng = np.random.default_rng(5)
        U0 = [np.asfortranarray(rng.standard_normal(solver.extents(j))) for j in range(S.n_sys)]
        outs = {j: np.zeros(int(np.prod(solver.extents(j)))) for j in range(S.n_sys)}
        page = 4096
        for a in list(U0) + list(outs.values()):
            nbytes = a.size * 8
            assert nbytes > 4 * page
            base = a.ctypes.data
            lo = (base + page - 1) // page * page           # whole pages inside the array
            hi = (base + nbytes) // page * page
            mid = (lo + hi) // 2 // page * page
            start, end = (lo, mid) if half == "first" else (mid, hi)
            assert int(cudart.cudaHostRegister(start, end - start, 0)) == 0
            regs.append(start)
        solver.set_state(U0)
        back = solver.get_state(out=outs)
        for j in range(S.n_sys):
            np.testing.assert_array_equal(back[j], U0[j])
    finally:
        for r in regs:
            cudart.cudaHostUnregister(r)
        solver.close()

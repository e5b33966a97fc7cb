"""smg_sumsq_noalloc: the reduction for hosts that must not allocate GPU memory.

Such a host (for example a MATLAB MEX gateway that only holds gpuArray buffers
owned by MATLAB's allocator) passes its own device input and output buffers;
the library keeps the partial sums in a fixed array of its own instead of
allocating.  The result must equal the ordinary, allocating reduction
(smg_state_sumsq) on the same data, and numpy's sum of squares on the host for
vectors with gaps between them, on consecutive calls that reuse the array.
Device buffers for the test are made with torch; the entry point itself
allocates nothing."""
import ctypes

import numpy as np
import pytest

import cases
from starmap_b200 import _lib, starmap_init
from starmap_b200.solver import GpuSolver, prepare

pytestmark = pytest.mark.gpu
REL_TOL = 1e-13


def padded(solver, U):
    """The handle's device layout of state U, as one host array (n_sys, cs)."""
    _, (s1, B1, B2, cs) = solver.layout()
    flat = np.zeros((solver.n_sys, cs))
    for j in range(solver.n_sys):
        e = [solver.extents(j)[d] for d in range(3)]
        # kernel axes: solver dimensions of extent > 1 first (column-major order kept)
        ke = [v for v in e if v > 1] + [v for v in e if v == 1]
        box = flat[j, :s1 * B1 * B2].reshape(B2, B1, s1)
        a = np.asarray(U[j]).reshape(ke, order="F")
        box[:ke[2], :ke[1], :ke[0]] = a.transpose(2, 1, 0)
    return flat, cs


def test_noalloc_sumsq_matches_allocating_reduction():
    torch = pytest.importorskip("torch")
    L = _lib.lib()
    par = starmap_init(cases.box3d_bc1_p2_full())
    S = prepare(par)
    fields = [(0.3, (1, 1, 1)), (1.0, (1, 1, 1))]
    solver = GpuSolver(S.n, S.bc, S.h, S.gt, S.Mx, S.My, S.Mz, fields, [0] * S.n_sys, 0, [-1] * S.n_sys,
                       decay_t=[1] * S.n_sys, decay_a=1)
    rng = np.random.default_rng(5)
    try:
        for call in range(2):   # two calls in a row share the library's scratch array
            U = [rng.standard_normal(solver.extents(j)) * (call + 1) for j in range(S.n_sys)]
            solver.set_state(U)
            ref = solver.state_sumsq()
            flat, cs = padded(solver, U)
            x = torch.from_numpy(flat).to("cuda")
            out = torch.full((S.n_sys,), float("nan"), dtype=torch.float64, device="cuda")
            stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
            rc = L.smg_sumsq_noalloc(ctypes.c_void_p(x.data_ptr()), S.n_sys, cs, cs,
                                     ctypes.c_void_p(out.data_ptr()), stream)
            assert rc == _lib.SMG_OK, L.smg_last_error(None)
            torch.cuda.synchronize()
            got = out.cpu().numpy()
            assert np.all(np.abs(got - ref) <= REL_TOL * np.abs(ref)), (call, got, ref)
    finally:
        solver.close()


def test_noalloc_sumsq_strided_vs_host_sum():
    """Vectors with gaps between them (stride > len): only the first len values
    of each vector count.  The gaps hold NaN and huge values, which would show
    in the result if they were read.  Checked against numpy's sum of squares on
    the host, on two calls in a row with different sizes."""
    torch = pytest.importorskip("torch")
    L = _lib.lib()
    rng = np.random.default_rng(9)
    for call, (ncomp, length, stride) in enumerate(((37, 5001, 5120), (1024, 777, 800))):
        host = np.full((ncomp, stride), np.nan)
        host[:, length + 1:] = 1e300
        host[:, :length] = rng.standard_normal((ncomp, length)) * (call + 1)
        x = torch.from_numpy(host).to("cuda")
        out = torch.full((ncomp,), float("nan"), dtype=torch.float64, device="cuda")
        rc = L.smg_sumsq_noalloc(ctypes.c_void_p(x.data_ptr()), ncomp, stride, length,
                                 ctypes.c_void_p(out.data_ptr()), None)
        assert rc == _lib.SMG_OK, L.smg_last_error(None)
        torch.cuda.synchronize()
        got = out.cpu().numpy()
        ref = np.sum(host[:, :length] * host[:, :length], axis=1)
        assert np.all(np.isfinite(got)), call
        assert np.all(np.abs(got - ref) <= REL_TOL * ref), (call, np.max(np.abs(got - ref) / ref))


def test_noalloc_sumsq_rejects_too_many_components():
    torch = pytest.importorskip("torch")
    L = _lib.lib()
    x = torch.zeros(8, dtype=torch.float64, device="cuda")
    out = torch.zeros(8, dtype=torch.float64, device="cuda")
    rc = L.smg_sumsq_noalloc(ctypes.c_void_p(x.data_ptr()), 1025, 1, 1, ctypes.c_void_p(out.data_ptr()), None)
    assert rc == _lib.SMG_EINVAL
    assert b"exceed the fixed scratch" in L.smg_last_error(None)

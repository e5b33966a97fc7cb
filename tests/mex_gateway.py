"""Test harness of the MEX gateway (matlab/starmap_solver_mex.c).

MATLAB and GNU Octave are not installed where this library is tested, so the
gateway is compiled with gcc against a test-only stand-in of the MATLAB C API
(tests/mex/mex.h, tests/mex/mex_stub.c), linked against libstarmap_gpu.so,
and called through ctypes with mxArrays built from the same host setup the
Python path uses -- the descriptor matlab/starmap_solver.m builds, with
MATLAB's 1-based field numbers.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = [os.path.join(ROOT, "matlab", "starmap_solver_mex.c"), os.path.join(HERE, "mex", "mex_stub.c")]
OUT = os.path.join(ROOT, "_build", "mex_gateway", "libstarmap_solver_mex_stub.so")


def build() -> str:
    from starmap_b200 import build as lib_build
    lib = lib_build.build()
    deps = SRC + [os.path.join(HERE, "mex", "mex.h"), os.path.join(ROOT, "include", "starmap_gpu.h"), lib]
    if os.path.exists(OUT) and all(os.path.getmtime(d) <= os.path.getmtime(OUT) for d in deps):
        return OUT
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    libdir = os.path.dirname(lib)
    cmd = ["gcc", "-std=c99", "-O2", "-Wall", "-Wextra", "-Werror", "-shared", "-fPIC",
           "-I", os.path.join(HERE, "mex"), "-I", os.path.join(ROOT, "include"), *SRC,
           "-L", libdir, "-lstarmap_gpu", "-Wl,-rpath," + libdir, "-o", OUT + ".tmp"]
    subprocess.run(cmd, check=True, capture_output=True, text=True)
    os.replace(OUT + ".tmp", OUT)
    return OUT


class Gateway:
    def __init__(self):
        L = C.CDLL(build())
        P = C.c_void_p
        L.stub_double.restype = P
        L.stub_double.argtypes = [C.c_size_t, C.POINTER(C.c_size_t), C.POINTER(C.c_double)]
        L.stub_cell.restype = P
        L.stub_cell.argtypes = [C.c_size_t]
        L.stub_string.restype = P
        L.stub_string.argtypes = [C.c_char_p]
        L.mxSetCell.argtypes = [P, C.c_size_t, P]
        L.mxGetCell.restype = P
        L.mxGetCell.argtypes = [P, C.c_size_t]
        L.stub_struct.restype = P
        L.stub_struct_set.argtypes = [P, C.c_char_p, P]
        L.stub_call.argtypes = [C.c_int, C.POINTER(P), C.c_int, C.POINTER(P)]
        L.stub_error.restype = C.c_char_p
        L.stub_error_id.restype = C.c_char_p
        L.mxGetPr.restype = C.POINTER(C.c_double)
        L.mxGetPr.argtypes = [P]
        L.mxGetNumberOfElements.restype = C.c_size_t
        L.mxGetNumberOfElements.argtypes = [P]
        L.mxGetNumberOfDimensions.restype = C.c_size_t
        L.mxGetNumberOfDimensions.argtypes = [P]
        L.mxGetDimensions.restype = C.POINTER(C.c_size_t)
        L.mxGetDimensions.argtypes = [P]
        self.L = L

    def array(self, a) -> int:
        a = np.asarray(a, dtype=np.float64)
        if a.ndim < 2:
            a = a.reshape(1, -1) if a.ndim == 1 else a.reshape(1, 1)
        dims = (C.c_size_t * a.ndim)(*a.shape)
        flat = np.ascontiguousarray(a.ravel(order="F"))
        return self.L.stub_double(a.ndim, dims, flat.ctypes.data_as(C.POINTER(C.c_double)))

    def string(self, s: str) -> int:
        return self.L.stub_string(s.encode())

    def cell(self, items) -> int:
        c = self.L.stub_cell(len(items))
        for i, it in enumerate(items):
            self.L.mxSetCell(c, i, it)
        return c

    def struct(self, fields: dict) -> int:
        s = self.L.stub_struct()
        for k, v in fields.items():
            assert self.L.stub_struct_set(s, k.encode(), v) == 0
        return s

    def to_numpy(self, a) -> np.ndarray:
        n = self.L.mxGetNumberOfElements(a)
        nd = self.L.mxGetNumberOfDimensions(a)
        dims = [self.L.mxGetDimensions(a)[k] for k in range(nd)]
        return np.ctypeslib.as_array(self.L.mxGetPr(a), shape=(n,)).copy().reshape(dims, order="F")

    def call(self, args, nlhs=2):
        """(None, outputs) or (error id, message)."""
        P = C.c_void_p
        plhs = (P * max(nlhs, 1))()
        prhs = (P * len(args))(*args)
        if self.L.stub_call(nlhs, plhs, len(args), prhs):
            return self.L.stub_error_id().decode(), self.L.stub_error().decode()
        return None, [plhs[i] for i in range(nlhs)]


def descriptor(G: Gateway, S, T, tables: dict, overrides=None) -> int:
    """The desc struct matlab/starmap_solver.m passes for host setup S and field table T."""
    one = lambda v: np.asarray([int(x) + 1 for x in v], dtype=np.float64)   # 0-based -> 1-based, -1 -> 0
    mode = tables["filter_mode"]
    n_sys = S.n_sys
    f = {
        "n": G.array(np.asarray(S.n, dtype=np.float64)), "bc": G.array(np.asarray(S.bc, dtype=np.float64)),
        "h": G.array(np.asarray(S.h, dtype=np.float64)),
        "gt": G.array(np.asarray(S.gt, dtype=np.float64).reshape(n_sys, 3)),
        "Mx": G.array(S.Mx), "My": G.array(S.My), "Mz": G.array(S.Mz),
        "fields": G.cell([G.array(np.asarray(v, dtype=np.float64)) for v, _ in T.fields]),
        "field_grid": G.array(np.asarray([g for _, g in T.fields], dtype=np.float64).reshape(-1, 3)),
        "sigma_t": G.array(one(tables["sigma_t"])), "decay_t": G.array(one(tables["decay_t"])),
        "source": G.array(one(tables["source"])),
        "sigma_a": G.array(float(tables["sigma_a"] + 1)), "decay_a": G.array(float(tables["decay_a"] + 1)),
        "filter_mode": G.array(float(mode)),
    }
    if mode:
        f["filter1"] = G.array(one(tables["filter1"]))
    if mode == 1:
        f["filter2"] = G.array(one(tables["filter2"]))
    for k, v in (overrides or {}).items():
        if v is None:
            f.pop(k, None)
        else:
            f[k] = v
    return G.struct(f)

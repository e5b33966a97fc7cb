"""Moment-system matrices of the P_N and SP_N closures.

Host-side tables consumed by the solver: ``(mom_order, Mx, My, Mz)`` for a
closure of order ``n_mom`` in ``dim`` dimensions.  They are the input of the
time-stepping path, produced the same way as ``starmap_closure_pn.m`` and
``starmap_closure_spn.m`` of StaRMAP v2.0 (including the 2D convention that the
solver's first axis is a singleton, so the x/y matrices are stored in My/Mz and
Mx is zero).  Every floating-point expression keeps the reference's operation
order so the tables agree to the last bit with what MATLAB/Octave builds.

Matrices are dense ``float64`` arrays of shape ``(n_sys, n_sys)``; ``mom_order``
is an ``int64`` vector (a one-element vector holding ``n_mom + 1`` in 1D, which
is the reference's scalar value).
"""
from __future__ import annotations

import numpy as np

__all__ = ["closure_pn", "closure_spn", "closure"]


def _D(l, m):
    # starmap_closure_pn.m:91-92
    return np.sqrt((l - m) * (l - m - 1) / (2 * l + 1) / (2 * l - 1))


def _F(l, m):
    # starmap_closure_pn.m:94-95
    return np.sqrt((l + m) * (l + m - 1) / (2 * l + 1) / (2 * l - 1))


def _B(l, m):
    # starmap_closure_pn.m:97-98
    return np.sqrt((l - m) * (l + m) / (2 * l + 1) / (2 * l - 1))


def _neg1pow(i):
    """(-1).^i for an integer vector, as float64."""
    return np.where(np.asarray(i) % 2 == 0, 1.0, -1.0)


def _tridiag_1d(n_mom):
    """1D moment matrix (starmap_closure_pn.m:29-42, identical in the SP_N file)."""
    n_sys = n_mom + 1
    Mz = np.zeros((n_sys, n_sys))
    for k in range(0, n_sys - 1):
        Mz[k + 1, k] = (k + 1) / (2 * k + 3)   # spdiags sub-diagonal
        Mz[k, k + 1] = (k + 1) / (2 * k + 1)   # spdiags super-diagonal
    z = np.zeros((n_sys, n_sys))
    return np.array([n_mom + 1], dtype=np.int64), z, z.copy(), Mz


def closure_pn(n_mom: int, dim: int):
    """P_N matrices; follows starmap_closure_pn.m:28-89."""
    n_mom = int(n_mom)
    if dim == 1:
        return _tridiag_1d(n_mom)
    if dim == 2:
        n_sys = (n_mom + 1) * (n_mom + 2) // 2
        Mx = np.zeros((n_sys, n_sys))
        My = np.zeros((n_sys, n_sys))
        for m in range(1, n_mom + 1):
            i = np.arange(1, m + 1)
            p = m * (m - 1) // 2 + i                      # 1-based rows
            v = _D(float(m), -m + 2.0 * (np.ceil(i / 2) - 1))
            Mx[p - 1, p + m - 1] = v
            s = _neg1pow(i)
            My[p - 1, (p + m - s.astype(np.int64)) - 1] = -s * v
            i = np.arange(1, m)
            if i.size:
                p = m * (m - 1) // 2 + i
                v = _F(float(m), -m + 2 + 2.0 * (np.ceil(i / 2) - 1))
                Mx[p - 1, p + m + 2 - 1] = -v
                s = _neg1pow(i)
                My[(p - s.astype(np.int64)) - 1, p + m + 2 - 1] = s * v
        r2 = np.sqrt(2.0)
        m = np.arange(1, n_mom + 1, 2)
        i = m * (m + 1) // 2
        Mx[i - 1, :] = r2 * Mx[i - 1, :]
        My[i - 1, :] = r2 * My[i - 1, :]
        m = np.arange(2, n_mom + 1, 2)
        i = (m + 1) * (m + 2) // 2
        Mx[:, i - 1] = r2 * Mx[:, i - 1]
        My[:, i - 1] = r2 * My[:, i - 1]
        Mx = (Mx + Mx.T) / 2
        My = (My + My.T) / 2
        # solver ordering: Mz = My; My = Mx; Mx = 0  (starmap_closure_pn.m:62)
        Mz, My, Mx = My, Mx, np.zeros((n_sys, n_sys))
        k = np.arange(1, n_sys + 1)
        order = np.ceil(np.sqrt(2 * k + 1 / 4) - 3 / 2).astype(np.int64)
        return order, Mx, My, Mz
    if dim == 3:
        n_sys = (n_mom + 1) ** 2
        Mx = np.zeros((n_sys, n_sys))
        My = np.zeros((n_sys, n_sys))
        Mz = np.zeros((n_sys, n_sys))
        for m in range(1, n_mom + 1):
            i = np.arange(1, 2 * m)
            p = (m - 1) ** 2 + i
            v = _F(float(m), m + 1 - np.ceil(i / 2))
            Mx[p - 1, p + 2 * m - 1 - 1] = v
            s = _neg1pow(i)
            My[p - 1, (p + 2 * m - 1 - s.astype(np.int64)) - 1] = -s * v
            v = _B(float(m), m - np.ceil(i / 2))
            Mz[p - 1, p + 2 * m + 1 - 1] = v
            i = np.arange(1, 2 * m - 2)
            if i.size:
                p = (m - 1) ** 2 + i
                v = _D(float(m), m - 1 - np.ceil(i / 2))
                Mx[p - 1, p + 2 * m + 3 - 1] = -v
                if m > 1:
                    p = p.copy(); i = i.copy()
                    p[-1] += 1
                    i[-1] += 1
                s = _neg1pow(i)
                My[p - 1, (p + 2 * m + 3 - s.astype(np.int64)) - 1] = -s * v
        r2 = np.sqrt(2.0)
        m = np.arange(1, n_mom + 1)
        i = m ** 2
        Mx[i - 1, :] = r2 * Mx[i - 1, :]
        My[i - 1, :] = r2 * My[i - 1, :]
        m = np.arange(2, n_mom + 1)
        i = (m + 1) ** 2
        Mx[:, i - 1] = r2 * Mx[:, i - 1]
        My[:, i - 1] = r2 * My[:, i - 1]
        Mx = (Mx + Mx.T) / 2
        My = (My + My.T) / 2
        Mz = Mz + Mz.T
        k = np.arange(1, n_sys + 1)
        order = np.ceil(np.sqrt(k.astype(np.float64)) - 1).astype(np.int64)
        return order, Mx, My, Mz
    raise ValueError("dim must be 1, 2 or 3")


def _spn_blocks(n_mom):
    """Shared SP_N coefficient vectors (starmap_closure_spn.m:48-53 / 68-73)."""
    nstar = int(np.ceil((n_mom + 1) / 2))
    i = np.arange(0, nstar).astype(np.float64)
    k = 2 * i * (2 * i - 1) / ((4 * i + 1) * (4 * i - 1))
    odd_tail = (i < nstar - 1) | (np.floor(n_mom / 2) * 2 < n_mom)
    l = 4 * i ** 2 / ((4 * i + 1) * (4 * i - 1)) + \
        (2 * i + 1) ** 2 / ((4 * i + 1) * (4 * i + 3)) * odd_tail
    m = 2 * (2 * i + 1) * (i + 1) / ((4 * i + 1) * (4 * i + 3))
    T = np.diag(l)
    if nstar > 1:
        T = T + np.diag(k[1:], -1) + np.diag(m[:-1], 1)
    # diag(k(2:end),-1)+diag(l)+diag(m(1:end-1),1): the three diagonals are
    # disjoint, so the sum order cannot change any entry.
    return nstar, T


def closure_spn(n_mom: int, dim: int):
    """SP_N matrices; follows starmap_closure_spn.m:31-87."""
    n_mom = int(n_mom)
    if dim == 1:
        return _tridiag_1d(n_mom)
    nstar, T = _spn_blocks(n_mom)
    evens = np.arange(0, n_mom + 1, 2)
    if dim == 2:
        Mx = np.zeros((3 * nstar, 3 * nstar))
        rows = nstar + 2 * np.arange(nstar)            # nstar+(1:nstar)*2-1, 0-based
        Mx[np.ix_(rows, np.arange(nstar))] = T
        Mx[np.arange(nstar), rows] = 1.0
        q = np.arange(2 * nstar)
        perm = np.concatenate([np.arange(nstar), nstar + (q ^ 1)])
        My = Mx[np.ix_(perm, perm)]
        Mz, My, Mx = My, Mx, np.zeros_like(Mx)
        order = np.concatenate([evens, np.repeat(evens + 1, 2)]).astype(np.int64)
        return order, Mx, My, Mz
    if dim == 3:
        Mx = np.zeros((4 * nstar, 4 * nstar))
        rows = nstar + 3 * np.arange(nstar)            # nstar+(1:nstar)*3-2, 0-based
        Mx[np.ix_(rows, np.arange(nstar))] = T
        Mx[np.arange(nstar), rows] = 1.0
        q = np.arange(3 * nstar)
        r = q % 3
        py = np.where(r == 0, q + 1, np.where(r == 1, q - 1, q))
        pz = np.where(r == 0, q + 2, np.where(r == 2, q - 2, q))
        My = Mx[np.ix_(np.concatenate([np.arange(nstar), nstar + py]),
                       np.concatenate([np.arange(nstar), nstar + py]))]
        Mz = Mx[np.ix_(np.concatenate([np.arange(nstar), nstar + pz]),
                       np.concatenate([np.arange(nstar), nstar + pz]))]
        order = np.concatenate([evens, np.repeat(evens + 1, 3)]).astype(np.int64)
        return order, Mx, My, Mz
    raise ValueError("dim must be 1, 2 or 3")


def closure(name: str, n_mom: int, dim: int):
    """Dispatch on ``par.closure`` ('P' or 'SP'), as starmap_init.m:64-69."""
    if name == "P":
        return closure_pn(n_mom, dim)
    if name == "SP":
        return closure_spn(n_mom, dim)
    raise ValueError("closure must be 'P' or 'SP'")

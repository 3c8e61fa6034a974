"""AO one-electron integrals over Cartesian Gaussians (host-side input).

std2 computes the AO overlap S, the dipole-length matrix, the velocity
(nabla) matrix and the angular-momentum (r x nabla) matrix before it calls
``stda`` and hands them over as packed lower triangles (``main.f:756-797``;
libcint for S/r/nabla ``libcint.f:19-352,653-756``, the old deck for
r x nabla ``intslvm.f:213-300``).  This module produces the same four
operators from a :class:`~stda_b200.molden.Molecule` with an Obara-Saika
recursion in numpy, vectorised over shell pairs of one angular-momentum class.

Sign and origin conventions (the ones the boundary expects):

* ``S[a,b]  = <a|b>``
* ``L[c,a,b] = -<a| r_c |b>`` with the origin at (0,0,0) (``libcint.f:326``:
  ``mu = -buf`` of ``cint1e_r_cart`` with ``env(2:4)=0``)
* ``V[c,a,b] = -<a| d/dr_c |b>``, derivative on the ket (``intslvm.f:150-153``,
  ``velo.f`` header: ``r7 = r7 - v``)
* ``M[c,a,b] = <a| (r x nabla)_c |b>``, origin (0,0,0), derivative on the ket
  (``intpack.f90:1207-1284`` ``opam``: ``v(1)=s2*(sy*s9-sz*s6)``).

V and M are antisymmetric; the packed form stores element (a,b) with a>=b,
as in the reference's scratch files read by ``ONETRI(-1,...)`` (``onetri.f:73-79``:
``B(I,J)=A(IJ)``, ``B(J,I)=-A(IJ)`` for I>J).
"""
from __future__ import annotations

import math

import numpy as np

from .molden import CART_ORDER, Molecule, _dfact

SCREEN = 1e-18   # drop primitive pairs whose Gaussian prefactor is below this


def _shell_table(mol: Molecule):
    """Per shell: atom, l, exps, primitive-normalised coefs, AO offset, comp norms."""
    out = []
    off = 0
    for s in mol.shells:
        fac = (math.pi / (2.0 * s.exps)) ** 1.5 * _dfact(2 * s.l - 1) / (4.0 * s.exps) ** s.l
        cprim = s.coefs / np.sqrt(fac)
        norms = []
        for (lx, ly, lz) in CART_ORDER[s.l]:
            L = s.l
            pref = math.pi ** 1.5 * _dfact(2 * lx - 1) * _dfact(2 * ly - 1) * _dfact(2 * lz - 1) / 2.0 ** L
            ss = np.sum(np.outer(cprim, cprim) / (s.exps[:, None] + s.exps[None, :]) ** (L + 1.5))
            norms.append(1.0 / math.sqrt(pref * ss))
        out.append((s.atom, s.l, s.exps, cprim, off, np.asarray(norms)))
        off += s.ncart
    return out, off


def _os_1d(la, lb, PA, PB, p):
    """1D Obara-Saika overlap table without the Gaussian prefactor.

    Returns E[..., i, j] for i<=la, j<=lb+1 (one extra ket power for the
    moment and derivative operators).
    """
    shp = PA.shape
    nb = lb + 2
    E = np.zeros(shp + (la + 1, nb))
    E[..., 0, 0] = 1.0
    inv2p = 0.5 / p
    # build along the ket first: E(0,j)
    for j in range(1, nb):
        E[..., 0, j] = PB * E[..., 0, j - 1]
        if j >= 2:
            E[..., 0, j] += (j - 1) * inv2p * E[..., 0, j - 2]
    for i in range(1, la + 1):
        for j in range(0, nb):
            v = PA * E[..., i - 1, j]
            if i >= 2:
                v = v + (i - 1) * inv2p * E[..., i - 2, j]
            if j >= 1:
                v = v + j * inv2p * E[..., i - 1, j - 1]
            E[..., i, j] = v
    return E


def ao_integrals(mol: Molecule, chunk: int = 20000):
    """Return (S, L, V, M) as dense arrays: (nao,nao), (3,nao,nao) x3."""
    shells, nao = _shell_table(mol)
    S = np.zeros((nao, nao))
    L = np.zeros((3, nao, nao))
    V = np.zeros((3, nao, nao))
    M = np.zeros((3, nao, nao))
    xyz = mol.xyz
    ns = len(shells)
    # group ordered shell pairs (sa >= sb) by (la, lb, npa, npb)
    groups = {}
    for a in range(ns):
        for b in range(a + 1):
            sa, sb = shells[a], shells[b]
            key = (sa[1], sb[1], len(sa[2]), len(sb[2]))
            groups.setdefault(key, []).append((a, b))
    for (la, lb, npa, npb), pairs in groups.items():
        for c0 in range(0, len(pairs), chunk):
            sub = pairs[c0:c0 + chunk]
            ia = np.array([p[0] for p in sub])
            ib = np.array([p[1] for p in sub])
            A = xyz[[shells[i][0] for i in ia]]           # (P,3)
            B = xyz[[shells[i][0] for i in ib]]
            al = np.stack([shells[i][2] for i in ia])     # (P,npa)
            be = np.stack([shells[i][2] for i in ib])     # (P,npb)
            ca = np.stack([shells[i][3] for i in ia])
            cb = np.stack([shells[i][3] for i in ib])
            a_ = al[:, :, None]
            b_ = be[:, None, :]
            p = a_ + b_                                     # (P,npa,npb)
            mu = a_ * b_ / p
            AB2 = np.sum((A - B) ** 2, axis=1)[:, None, None]
            K = np.exp(-mu * AB2)
            keep = (K > SCREEN).any(axis=(1, 2))
            if not keep.any():
                continue
            ia, ib, A, B = ia[keep], ib[keep], A[keep], B[keep]
            a_, b_, p, K = a_[keep], b_[keep], p[keep], K[keep]
            w = ca[keep][:, :, None] * cb[keep][:, None, :] * K * (math.pi / p) ** 1.5
            P = (a_[..., None] * A[:, None, None, :] + b_[..., None] * B[:, None, None, :]) / p[..., None]
            tabs = []
            for d in range(3):
                PA = P[..., d] - A[:, None, None, d]
                PB = P[..., d] - B[:, None, None, d]
                E = _os_1d(la, lb, PA, PB, p)             # (P,npa,npb,la+1,lb+2)
                Bd = B[:, None, None, d][..., None, None]
                Mom = np.empty_like(E[..., :lb + 1])
                Mom[...] = E[..., 1:lb + 2] + Bd * E[..., :lb + 1]
                Der = np.empty_like(Mom)
                bb = (2.0 * b_)[..., None, None]
                Der[...] = -bb * E[..., 1:lb + 2]
                for j in range(1, lb + 1):
                    Der[..., j] += j * E[..., j - 1]
                tabs.append((E[..., :lb + 1], Mom, Der))
            ncomp_a = CART_ORDER[la]
            ncomp_b = CART_ORDER[lb]
            offa = np.array([shells[i][4] for i in ia])
            offb = np.array([shells[i][4] for i in ib])
            na = np.stack([shells[i][5] for i in ia])
            nb = np.stack([shells[i][5] for i in ib])
            for ka, (ax, ay, az) in enumerate(ncomp_a):
                for kb, (bx, by, bz) in enumerate(ncomp_b):
                    Sx, Mx, Dx = (t[..., ax, bx] for t in tabs[0])
                    Sy, My, Dy = (t[..., ay, by] for t in tabs[1])
                    Sz, Mz, Dz = (t[..., az, bz] for t in tabs[2])
                    nrm = na[:, ka] * nb[:, kb]

                    def red(x):
                        return np.sum(w * x, axis=(1, 2)) * nrm

                    s_ = red(Sx * Sy * Sz)
                    rx = red(Mx * Sy * Sz)
                    ry = red(Sx * My * Sz)
                    rz = red(Sx * Sy * Mz)
                    dx = red(Dx * Sy * Sz)
                    dy = red(Sx * Dy * Sz)
                    dz = red(Sx * Sy * Dz)
                    lx = red(Sx * (My * Dz - Mz * Dy))
                    ly = red(Sy * (Mz * Dx - Mx * Dz))
                    lz = red(Sz * (Mx * Dy - My * Dx))
                    r_ = offa + ka
                    c_ = offb + kb
                    S[r_, c_] = s_
                    S[c_, r_] = s_
                    for d, v in enumerate((rx, ry, rz)):
                        L[d, r_, c_] = -v
                        L[d, c_, r_] = -v
                    for d, v in enumerate((dx, dy, dz)):
                        V[d, r_, c_] = -v
                        V[d, c_, r_] = v
                    for d, v in enumerate((lx, ly, lz)):
                        M[d, r_, c_] = v
                        M[d, c_, r_] = -v
    # exact antisymmetry on the diagonal
    for d in range(3):
        np.fill_diagonal(V[d], 0.0)
        np.fill_diagonal(M[d], 0.0)
    return S, L, V, M


def pack_lower(mat: np.ndarray) -> np.ndarray:
    """Row-wise packed lower triangle: k enumerates (i, j<=i), value mat[i, j].

    This is the layout of the reference's ``sint``/``xlint``/... files
    (``libcint.f:212-240`` with ``lin8``; ``stda.f:2174-2181``).
    """
    n = mat.shape[-1]
    ii, jj = np.tril_indices(n)
    order = np.lexsort((jj, ii))
    return np.ascontiguousarray(mat[..., ii[order], jj[order]])


def unpack_lower(packed: np.ndarray, n: int, antisym: bool = False) -> np.ndarray:
    """Inverse of :func:`pack_lower` (``onetri.f:62-80`` BLOWSY)."""
    ii, jj = np.tril_indices(n)
    order = np.lexsort((jj, ii))
    ii, jj = ii[order], jj[order]
    out = np.zeros(packed.shape[:-1] + (n, n))
    out[..., ii, jj] = packed
    if antisym:
        out[..., jj, ii] = -packed
        d = np.arange(n)
        out[..., d, d] = 0.0
    else:
        out[..., jj, ii] = packed
    return out

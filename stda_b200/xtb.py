"""xTB input path: the ``wfn.xtb`` wavefunction file and the ``-xtb`` keyword
defaults (sTDA-xTB).

``wfn.xtb`` is a Fortran unformatted sequential file (4-byte record markers)
that xtb4stda writes and std2 reads in ``readxtb0`` / ``readxtb``
(``readxtb.f:38-200``).  Records, in order:

1. ``imethod`` (1 restricted, 2 unrestricted)
2. ``ncent, nbf, nmo, nprims``
3. ``ncent`` records of the two-character atom names
4. per atom: three records x, y, z (real*8, Bohr) and one record Z (integer)
5. ``nprims`` one-integer records each of ``ipty``, then ``ipat``, then ``ipao``
6. one record of the ``nprims`` exponents, one of the contraction coefficients
7. restricted: ``occ(nmo)``, ``eps(nmo)``, ``C(nbf*nmo)`` (column-major);
   unrestricted: alpha ``occ``, ``eps``, beta ``occ``, ``eps`` (``nmo`` each,
   the file's ``nmo`` is per spin), then alpha ``C``, beta ``C``.

The primitive arrays are exactly what the engine's device integrals take
(``std2g_load_prims``); the coefficients already carry every normalisation
(``fnorm`` = 1 for xTB input, ``main.f:832-838``).  Unrestricted files load as
UKS (``std2g_set_spins``).

``-xtb`` sets ax = 0.5, alpha = 2.0, beta = 4.0 and switches the K-shift of
the diagonal on with shftmax = 0.5 eV, shftwidth = 0.1 eV, shftsteep = 4.0
(``main.f:202-219``).
"""
from __future__ import annotations

import struct
from dataclasses import dataclass

import numpy as np

from .engine import Keywords, Primitives


@dataclass
class XtbWavefunction:
    imethod: int
    atnam: list
    xyz: np.ndarray          # (ncent, 3) Bohr
    Z: np.ndarray            # (ncent,) int
    nbf: int
    prims: Primitives
    C: np.ndarray            # (nbf, nmo) restricted; (2, nbf, nmo) unrestricted
    eps: np.ndarray          # (nmo,) or (2, nmo)
    occ: np.ndarray

    @property
    def ncent(self) -> int:
        return len(self.Z)

    def xyz4(self) -> np.ndarray:
        """(ncent, 4) rows x, y, z, Z: Fortran xyz(4, ncent)."""
        return np.hstack([self.xyz, self.Z[:, None].astype(np.float64)])


def xtb_keywords(**overrides) -> Keywords:
    """Keywords with the ``-xtb`` defaults of ``main.f:202-219``."""
    kw = dict(ax=0.5, alpha_k=2.0, beta_j=4.0, kshift=True, shftmax=0.5, shftwidth=0.1,
              shftsteep=4.0)
    kw.update(overrides)
    return Keywords(**kw)


class _Records:
    """Sequential reader of gfortran unformatted records (a negative leading
    marker continues the record in the next subrecord)."""

    def __init__(self, data: bytes):
        self.data = data
        self.pos = 0

    def next(self) -> bytes:
        out = b""
        while True:
            if self.pos + 4 > len(self.data):
                raise ValueError("wfn.xtb: unexpected end of file")
            (m,) = struct.unpack_from("<i", self.data, self.pos)
            n = abs(m)
            start = self.pos + 4
            if start + n + 4 > len(self.data):
                raise ValueError("wfn.xtb: truncated record")
            out += self.data[start:start + n]
            (tail,) = struct.unpack_from("<i", self.data, start + n)
            if abs(tail) != n:
                raise ValueError("wfn.xtb: record markers disagree")
            self.pos = start + n + 4
            if m >= 0:
                return out

    def ints(self, count=None):
        r = self.next()
        v = np.frombuffer(r, dtype="<i4")
        if count is not None and len(v) != count:
            raise ValueError(f"wfn.xtb: expected {count} integers, found {len(v)}")
        return v

    def reals(self, count):
        r = self.next()
        v = np.frombuffer(r, dtype="<f8")
        if len(v) != count:
            raise ValueError(f"wfn.xtb: expected {count} reals, found {len(v)}")
        return v.copy()


def read_wfn_xtb(path: str) -> XtbWavefunction:
    """Read ``wfn.xtb`` as ``readxtb0`` + ``readxtb`` do (``readxtb.f:38-200``)."""
    with open(path, "rb") as fh:
        rec = _Records(fh.read())
    imethod = int(rec.ints(1)[0])
    if imethod not in (1, 2):
        raise ValueError(f"wfn.xtb: imethod {imethod} is neither 1 (RKS) nor 2 (UKS)")
    ncent, nbf, nmo, nprims = (int(x) for x in rec.ints(4))
    if min(ncent, nbf, nmo, nprims) <= 0:
        raise ValueError("wfn.xtb: read error (zero dimension)")
    atnam = [rec.next().decode("ascii", "replace").strip() for _ in range(ncent)]
    xyz = np.zeros((ncent, 3))
    Z = np.zeros(ncent, dtype=np.int64)
    for i in range(ncent):
        for j in range(3):
            xyz[i, j] = rec.reals(1)[0]
        Z[i] = rec.ints(1)[0]
        if Z[i] < 1:
            atnam[i] = "xx"
    ipty = np.array([rec.ints(1)[0] for _ in range(nprims)], dtype=np.int32)
    ipat = np.array([rec.ints(1)[0] for _ in range(nprims)], dtype=np.int32)
    ipao = np.array([rec.ints(1)[0] for _ in range(nprims)], dtype=np.int32)
    if ipty.min() < 1 or ipty.max() > 20:
        raise ValueError("wfn.xtb: functions beyond f in the basis (ipty > 20)")
    exip = rec.reals(nprims)
    cxip = rec.reals(nprims)
    prims = Primitives(ipty, ipao, ipat, exip, cxip)
    if imethod == 1:
        occ = rec.reals(nmo)
        eps = rec.reals(nmo)
        C = rec.reals(nbf * nmo).reshape(nmo, nbf).T.copy()
    else:
        occ_a, eps_a = rec.reals(nmo), rec.reals(nmo)
        occ_b, eps_b = rec.reals(nmo), rec.reals(nmo)
        Ca = rec.reals(nbf * nmo).reshape(nmo, nbf).T
        Cb = rec.reals(nbf * nmo).reshape(nmo, nbf).T
        occ, eps, C = np.stack([occ_a, occ_b]), np.stack([eps_a, eps_b]), np.stack([Ca, Cb])
    return XtbWavefunction(imethod, atnam, xyz, Z, nbf, prims, C, eps, occ)


def write_wfn_xtb(path: str, wf: XtbWavefunction) -> None:
    """Write ``wfn.xtb`` in the record layout ``readxtb`` reads."""
    def rec(b: bytes):
        return struct.pack("<i", len(b)) + b + struct.pack("<i", len(b))

    i4 = lambda *v: np.asarray(v, dtype="<i4").tobytes()  # noqa: E731
    f8 = lambda v: np.ascontiguousarray(v, dtype="<f8").tobytes()  # noqa: E731
    pr = wf.prims
    nmo = wf.C.shape[-1]
    out = [rec(i4(wf.imethod)), rec(i4(wf.ncent, wf.nbf, nmo, pr.nprims))]
    out += [rec(("%-2s" % n)[:2].encode("ascii")) for n in wf.atnam]
    for i in range(wf.ncent):
        out += [rec(f8([wf.xyz[i, j]])) for j in range(3)] + [rec(i4(int(wf.Z[i])))]
    for arr in (pr.ipty, pr.ipat, pr.ipao):
        out += [rec(i4(int(v))) for v in arr]
    out += [rec(f8(pr.exip)), rec(f8(pr.cxip))]
    if wf.imethod == 1:
        out += [rec(f8(wf.occ)), rec(f8(wf.eps)), rec(f8(np.asarray(wf.C).T.ravel()))]
    else:
        out += [rec(f8(wf.occ[0])), rec(f8(wf.eps[0])), rec(f8(wf.occ[1])), rec(f8(wf.eps[1])),
                rec(f8(np.asarray(wf.C[0]).T.ravel())), rec(f8(np.asarray(wf.C[1]).T.ravel()))]
    with open(path, "wb") as fh:
        fh.write(b"".join(out))


def from_molecule(mol) -> XtbWavefunction:
    """A restricted ``wfn.xtb`` image of a molecule with MOs (test fixtures)."""
    from .engine import primitives
    from .molden import ELEMENT_SYMBOLS
    names = [ELEMENT_SYMBOLS[int(z)] if int(z) < len(ELEMENT_SYMBOLS) else "xx" for z in mol.Z]
    return XtbWavefunction(1, names, np.asarray(mol.xyz, dtype=np.float64),
                           np.asarray(mol.Z, dtype=np.int64), mol.nao, primitives(mol),
                           np.asarray(mol.C, dtype=np.float64), np.asarray(mol.eps, dtype=np.float64),
                           np.asarray(mol.occ, dtype=np.float64))


def load_xtb(engine, wf: XtbWavefunction) -> None:
    """Load an xTB wavefunction; the AO integrals are formed on the device from
    its primitive list (std2g_load_prims).  Unrestricted input (imethod 2) is
    loaded as the alpha MOs followed by the beta MOs and marked with their
    spins (std2g_set_spins), as ``main.f:729-738`` sets ``ccspin``."""
    if wf.imethod == 1:
        engine.load_prims(wf.xyz4(), wf.C, wf.eps, wf.occ, wf.prims)
        return
    nmo = wf.C.shape[-1]
    C2 = np.hstack([wf.C[0], wf.C[1]])
    engine.load_prims(wf.xyz4(), C2, np.concatenate([wf.eps[0], wf.eps[1]]),
                      np.concatenate([wf.occ[0], wf.occ[1]]), wf.prims)
    engine.set_spins(np.concatenate([np.ones(nmo, dtype=np.int32),
                                     np.full(nmo, 2, dtype=np.int32)]))

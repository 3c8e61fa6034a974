"""Molden reader/writer for the host side of the engine (Cartesian GTOs).

This mirrors what std2 reads before it calls ``stda``: atoms (charge and
coordinates in Bohr), contracted Cartesian Gaussian shells, MO coefficients,
orbital energies and occupations (``readbasmold.f:217-740``).  The engine's
boundary takes exactly those arrays, so the reader fixes the same conventions:

* ``[Atoms] Angs`` coordinates are divided by 0.52917721092 (``readbasmold.f:270``).
* Every Cartesian component of every contraction is normalised to unit self
  overlap.  This is what ``-sty 3`` (TeraChem/Gaussian style) produces: the
  primitive normalisation of ``readbasmold.f:355-378`` followed by
  ``normalize(.true.,...)`` (``normalize.f:23-80``, ``xlinf = 1`` for a
  Cartesian basis).
* ``sp`` shells are split into an s and a p contraction with shared exponents
  (``readbasmold.f:330-366``).
* Component order inside a shell is the molden order (p: x y z; d: xx yy zz
  xy xz yz; f: xxx yyy zzz xyy xxy xxz xzz yzz yyz xyz).  std2 reorders f
  coefficients internally (``readbasmold.f:585-600``); here the AO order of the
  MO coefficients and of the integrals is the molden order throughout, which
  is equivalent.
* MO coefficients omitted in the file (TeraChem prints non-zero ones only) are
  zero (``readbasmold.f:606-628``).

Cartesian closed-shell (RKS) and open-shell (UKS) files are read: a file
with ``Spin= Beta`` MOs sets ``Molecule.csp`` (1 alpha / 2 beta per MO), which
the engine takes through ``std2g_set_spins`` (the reference dispatches such
files to ``sutda``, ``main.f:933``).  Spherical inputs raise ``ValueError``.
"""
from __future__ import annotations

import math
import re
from dataclasses import dataclass, field

import numpy as np

BOHR_ANGSTROM = 0.52917721092

# Cartesian exponents (lx, ly, lz) per shell type, molden order.
CART_ORDER = {
    0: [(0, 0, 0)],
    1: [(1, 0, 0), (0, 1, 0), (0, 0, 1)],
    2: [(2, 0, 0), (0, 2, 0), (0, 0, 2), (1, 1, 0), (1, 0, 1), (0, 1, 1)],
    3: [(3, 0, 0), (0, 3, 0), (0, 0, 3), (1, 2, 0), (2, 1, 0), (2, 0, 1),
        (1, 0, 2), (0, 1, 2), (0, 2, 1), (1, 1, 1)],
}
L_OF = {"s": 0, "p": 1, "d": 2, "f": 3}

ELEMENT_SYMBOLS = [
    "X", "H", "He", "Li", "Be", "B", "C", "N", "O", "F", "Ne", "Na", "Mg", "Al",
    "Si", "P", "S", "Cl", "Ar",
]


def _dfact(n: int) -> float:
    """(n)!! with (-1)!! = 1."""
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def component_norm(alphas: np.ndarray, coefs: np.ndarray, lmn) -> float:
    """Factor that makes sum_k c_k x^l y^m z^n exp(-a_k r^2) unit-normalised.

    Self overlap follows ``normalize.f:47-68``:
    pi^1.5 (2l-1)!!(2m-1)!!(2n-1)!! / 2^L * sum_kl c_k c_l / (a_k+a_l)^(L+1.5).
    """
    lx, ly, lz = lmn
    L = lx + ly + lz
    pref = math.pi ** 1.5 * _dfact(2 * lx - 1) * _dfact(2 * ly - 1) * _dfact(2 * lz - 1) / 2.0 ** L
    s = np.sum(np.outer(coefs, coefs) / (alphas[:, None] + alphas[None, :]) ** (L + 1.5))
    return 1.0 / math.sqrt(pref * s)


@dataclass
class Shell:
    atom: int            # 0-based atom index
    l: int
    exps: np.ndarray     # primitive exponents
    coefs: np.ndarray    # contraction coefficients as written in the file

    @property
    def ncart(self) -> int:
        return (self.l + 1) * (self.l + 2) // 2


@dataclass
class Molecule:
    Z: np.ndarray                 # (ncent,) nuclear charges (int)
    xyz: np.ndarray               # (ncent, 3) Bohr
    shells: list = field(default_factory=list)
    C: np.ndarray | None = None   # (nao, nmo) MO coefficients, column = MO
    eps: np.ndarray | None = None
    occ: np.ndarray | None = None
    title: str = ""
    csp: np.ndarray | None = None  # spin of each MO (1 alpha, 2 beta); None: restricted

    @property
    def ncent(self) -> int:
        return len(self.Z)

    @property
    def nao(self) -> int:
        return sum(s.ncart for s in self.shells)

    def iaoat(self) -> np.ndarray:
        """AO -> atom map, 0-based (``intslvm.f:71-74``)."""
        out = []
        for s in self.shells:
            out += [s.atom] * s.ncart
        return np.asarray(out, dtype=np.int32)

    def xyz4(self) -> np.ndarray:
        """(4, ncent) column-major-style array: x, y, z (Bohr) and Z."""
        return np.vstack([self.xyz.T, self.Z[None, :].astype(np.float64)])

    def ao_functions(self):
        """Per AO: (atom, (lx,ly,lz), exps, normalised primitive coefficients)."""
        out = []
        for s in self.shells:
            # primitive normalisation (readbasmold.f:355-378): divide by the
            # square root of <x^L g|x^L g> = (pi/2a)^1.5 (2L-1)!! / (4a)^L
            fac = (math.pi / (2.0 * s.exps)) ** 1.5 * _dfact(2 * s.l - 1) / (4.0 * s.exps) ** s.l
            cprim = s.coefs / np.sqrt(fac)
            for lmn in CART_ORDER[s.l]:
                # normalize.f:23-80 rescales each Cartesian component's
                # contraction to unit self overlap (Cartesian basis: xlinf=1)
                c = cprim * component_norm(s.exps, cprim, lmn)
                out.append((s.atom, lmn, s.exps, c))
        return out


def _ffloat(tok: str) -> float:
    return float(tok.replace("D", "E").replace("d", "e"))


def read_molden(path: str) -> Molecule:
    """Read a Cartesian closed-shell molden file (``-sty 3`` conventions)."""
    with open(path) as fh:
        lines = fh.read().splitlines()
    low = [ln.strip().lower() for ln in lines]

    def find(tag):
        for i, ln in enumerate(low):
            if ln.startswith(tag):
                return i
        raise ValueError(f"{tag} section missing in {path}")

    # [Atoms]
    ia = find("[atoms]")
    unit = lines[ia].split()
    scale = 1.0 / BOHR_ANGSTROM
    if len(unit) > 1 and unit[1].upper().startswith("AU"):
        scale = 1.0
    Z, xyz = [], []
    i = ia + 1
    while i < len(lines) and lines[i].strip() and not lines[i].strip().startswith("["):
        tok = lines[i].split()
        Z.append(int(tok[2]))
        xyz.append([_ffloat(t) * scale for t in tok[3:6]])
        i += 1
    Z = np.asarray(Z, dtype=np.int32)
    xyz = np.asarray(xyz, dtype=np.float64)

    if any(ln.startswith("[5d") or ln.startswith("[7f") or ln.startswith("[9g") for ln in low):
        raise ValueError("spherical molden basis is not supported (Cartesian only)")

    # [GTO]
    ig = find("[gto]")
    shells = []
    i = ig + 1
    atom = -1
    while i < len(lines):
        s = lines[i].strip()
        if s.startswith("["):
            break
        tok = s.split()
        if not tok:
            i += 1
            continue
        if len(tok) == 2 and tok[0].isdigit():
            atom = int(tok[0]) - 1
            i += 1
            continue
        kind = tok[0].lower()
        if kind in ("s", "p", "d", "f", "sp"):
            nprim = int(tok[1])
            rows = [lines[i + 1 + k].split() for k in range(nprim)]
            exps = np.array([_ffloat(r[0]) for r in rows])
            if kind == "sp":
                cs = np.array([_ffloat(r[1]) for r in rows])
                cp = np.array([_ffloat(r[2]) for r in rows])
                shells.append(Shell(atom, 0, exps, cs))
                shells.append(Shell(atom, 1, exps.copy(), cp))
            else:
                cc = np.array([_ffloat(r[1]) for r in rows])
                shells.append(Shell(atom, L_OF[kind], exps, cc))
            i += 1 + nprim
            continue
        if kind in ("g", "h"):
            raise ValueError("g/h shells are not supported")
        i += 1
    mol = Molecule(Z=Z, xyz=xyz, shells=shells)
    nao = mol.nao

    # [MO]
    im = find("[mo]")
    eps, occ, cols, spin = [], [], [], []
    cur = None
    i = im + 1
    while i < len(lines):
        s = lines[i].strip()
        if s.startswith("["):
            break
        if "=" in s:
            key, val = [t.strip() for t in s.split("=", 1)]
            k = key.lower()
            if k == "ene":
                if cur is not None:
                    cols.append(cur)
                cur = np.zeros(nao)
                eps.append(_ffloat(val))
            elif k == "occup":
                occ.append(_ffloat(val))
            elif k == "spin":
                spin.append(2 if val.lower().startswith("beta") else 1)
        else:
            tok = s.split()
            if len(tok) == 2 and re.fullmatch(r"\d+", tok[0]):
                idx = int(tok[0])
                if 1 <= idx <= nao:
                    cur[idx - 1] = _ffloat(tok[1])
        i += 1
    if cur is not None:
        cols.append(cur)
    mol.C = np.ascontiguousarray(np.array(cols).T)
    mol.eps = np.asarray(eps, dtype=np.float64)
    mol.occ = np.asarray(occ, dtype=np.float64)
    if mol.C.shape[1] != len(mol.eps) or len(mol.occ) != len(mol.eps):
        raise ValueError("inconsistent [MO] section")
    if 2 in spin:
        if len(spin) != len(mol.eps):
            raise ValueError("inconsistent Spin= lines in the [MO] section")
        mol.csp = np.asarray(spin, dtype=np.int32)
    return mol


def write_molden(mol: Molecule, path: str, title: str = "") -> None:
    """Write ``mol`` as a Cartesian molden file readable with ``-sty 3``."""
    out = ["[Molden Format]"]
    if title:
        out += ["[Title]", title]
    out.append("[Atoms] AU")
    for a in range(mol.ncent):
        sym = ELEMENT_SYMBOLS[int(mol.Z[a])] if int(mol.Z[a]) < len(ELEMENT_SYMBOLS) else "X"
        x, y, z = mol.xyz[a]
        out.append(f"{sym:<3s}{a + 1:6d}{int(mol.Z[a]):4d} {x:20.12f}{y:20.12f}{z:20.12f}")
    out.append("[GTO]")
    by_atom = {}
    for s in mol.shells:
        by_atom.setdefault(s.atom, []).append(s)
    letters = "spdf"
    for a in range(mol.ncent):
        out.append(f"  {a + 1} 0")
        for s in by_atom.get(a, []):
            out.append(f"  {letters[s.l]} {len(s.exps)} 1.00")
            for e, c in zip(s.exps, s.coefs):
                out.append(f"  {e:.10e} {c:.10e}")
        out.append(" ")
    out.append("[MO]")
    for m in range(mol.C.shape[1]):
        out.append(" Sym=  1")
        out.append(f" Ene= {mol.eps[m]:.15e}")
        beta = mol.csp is not None and int(mol.csp[m]) == 2
        out.append(" Spin= Beta" if beta else " Spin= Alpha")
        out.append(f" Occup= {mol.occ[m]:.6f}")
        col = mol.C[:, m]
        for k in range(mol.nao):
            out.append(f"{k + 1:6d} {col[k]:.15e}")
    with open(path, "w") as fh:
        fh.write("\n".join(out) + "\n")

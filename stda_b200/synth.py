"""Seeded synthetic molecules for the sTDA workloads (host-side input).

No public dataset is involved: every workload is a synthetic molecule with a
minimal Gaussian basis whose MO coefficients are C = S^-1/2 Q with Q a seeded
Haar-random orthogonal matrix, and whose orbital energies are sorted uniform
draws (occupied in [-0.8,-0.2] Eh, virtual in [0.0,0.6] Eh).  Löwdin MOs are
then exactly Q, so transition charges are those of random orthonormal
orbitals.

* :func:`benzene`        C6H6, ring C-C 1.39 A, C-H 1.09 A, STO-3G (36 AOs)
* :func:`graphene_flake` C_{6n^2}H_{6n} (n=8: C384H48), lattice 1.42 A, C-H
  1.09 A, minimal valence basis (C 2s2p from STO-3G's 2sp shell, H 1s):
  4*384+48 = 1584 AOs
* :func:`chain`          a C/N/O/H zig-zag chain, STO-3G
* :func:`random_molecule` a compact C/N/O/H cluster of a given size (batches)
"""
from __future__ import annotations

import math

import numpy as np

from .integrals import ao_integrals
from .molden import BOHR_ANGSTROM, Molecule, Shell

# STO-3G contraction coefficients (shared by first-row atoms) and exponents.
_C1S = np.array([0.15432897, 0.53532814, 0.44463454])
_C2S = np.array([-0.09996723, 0.39951283, 0.70011547])
_C2P = np.array([0.15591627, 0.60768372, 0.39195739])
_STO3G = {
    1: dict(s1=[3.42525091, 0.62391373, 0.16885540]),
    6: dict(s1=[71.6168370, 13.0450960, 3.5305122], sp=[2.9412494, 0.6834831, 0.2222899]),
    7: dict(s1=[99.1061690, 18.0523120, 4.8856602], sp=[3.7804559, 0.8784966, 0.2857144]),
    8: dict(s1=[130.7093200, 23.8088610, 6.4436083], sp=[5.0331513, 1.1695961, 0.3803890]),
}


def basis_shells(Z, valence_only=False):
    """Shells for the atoms with charges ``Z`` (STO-3G or its valence part)."""
    shells = []
    for a, z in enumerate(Z):
        d = _STO3G[int(z)]
        if int(z) == 1:
            shells.append(Shell(a, 0, np.array(d["s1"]), _C1S.copy()))
            continue
        if not valence_only:
            shells.append(Shell(a, 0, np.array(d["s1"]), _C1S.copy()))
        shells.append(Shell(a, 0, np.array(d["sp"]), _C2S.copy()))
        shells.append(Shell(a, 1, np.array(d["sp"]), _C2P.copy()))
    return shells


def haar_orthogonal(n, rng):
    """Haar-random orthogonal matrix: QR of a Gaussian matrix, sign-fixed."""
    g = rng.standard_normal((n, n))
    q, r = np.linalg.qr(g)
    return q * np.sign(np.diag(r))[None, :]


def attach_mos(mol: Molecule, nocc: int, seed: int, ints=None):
    """C = S^-1/2 Q, sorted uniform orbital energies, closed-shell occupations."""
    rng = np.random.default_rng(seed)
    S = (ints if ints is not None else ao_integrals(mol))[0]
    e, U = np.linalg.eigh(S)
    Sm12 = (U / np.sqrt(e)) @ U.T
    n = mol.nao
    Q = haar_orthogonal(n, rng)
    mol.C = Sm12 @ Q
    eo = np.sort(rng.uniform(-0.8, -0.2, nocc))
    ev = np.sort(rng.uniform(0.0, 0.6, n - nocc))
    mol.eps = np.concatenate([eo, ev])
    mol.occ = np.concatenate([np.full(nocc, 2.0), np.zeros(n - nocc)])
    return mol


def _ang(x):
    return np.asarray(x, dtype=np.float64) / BOHR_ANGSTROM


def benzene(seed: int = 0, with_ints=False):
    """Config-0 molecule: C6H6 with STO-3G (36 AOs), 21 occupied MOs."""
    cc, ch = 1.39, 1.09
    xyz, Z = [], []
    for k in range(6):
        t = math.pi / 3 * k
        xyz.append([cc * math.cos(t), cc * math.sin(t), 0.0])
        Z.append(6)
    for k in range(6):
        t = math.pi / 3 * k
        xyz.append([(cc + ch) * math.cos(t), (cc + ch) * math.sin(t), 0.0])
        Z.append(1)
    Z = np.array(Z, dtype=np.int32)
    mol = Molecule(Z=Z, xyz=_ang(xyz), shells=basis_shells(Z), title="benzene C6H6 STO-3G")
    ints = ao_integrals(mol)
    attach_mos(mol, 21, seed, ints)
    return (mol, ints) if with_ints else mol


def flake_geometry(n: int):
    """Hexagonal graphene flake C_{6n^2}H_{6n} (coronene series), Angstrom."""
    a = 1.42
    # hexagon centres on a triangular lattice (axial coordinates)
    cen = []
    for q in range(-(n - 1), n):
        for r in range(-(n - 1), n):
            if abs(q + r) <= n - 1:
                x = math.sqrt(3) * a * (q + r / 2.0)
                y = 1.5 * a * r
                cen.append((x, y))
    pts = {}
    for (x, y) in cen:
        for k in range(6):
            t = math.pi / 6 + math.pi / 3 * k
            px, py = x + a * math.cos(t), y + a * math.sin(t)
            key = (round(px, 4), round(py, 4))
            pts[key] = (px, py)
    C = np.array(sorted(pts.values()))
    d = np.sqrt(((C[:, None, :] - C[None, :, :]) ** 2).sum(-1))
    nb = ((d < a * 1.1) & (d > 0.1)).sum(1)
    H = []
    for i in np.nonzero(nb == 2)[0]:
        js = np.nonzero((d[i] < a * 1.1) & (d[i] > 0.1))[0]
        v = 2 * C[i] - C[js[0]] - C[js[1]]
        v /= np.linalg.norm(v)
        H.append(C[i] + 1.09 * v)
    C3 = np.hstack([C, np.zeros((len(C), 1))])
    H3 = np.hstack([np.array(H), np.zeros((len(H), 1))])
    return C3, H3


def graphene_flake(n: int = 8, nocc: int | None = None, seed: int = 1, with_ints=False):
    """Config-1 molecule (n=8): C384H48, minimal valence basis, 780 occ. MOs."""
    C3, H3 = flake_geometry(n)
    Z = np.array([6] * len(C3) + [1] * len(H3), dtype=np.int32)
    mol = Molecule(Z=Z, xyz=_ang(np.vstack([C3, H3])), shells=basis_shells(Z, valence_only=True),
                   title=f"graphene flake C{len(C3)}H{len(H3)} valence minimal basis")
    if nocc is None:
        nocc = 780 if n == 8 else (4 * len(C3) + len(H3)) // 2
    ints = ao_integrals(mol)
    attach_mos(mol, nocc, seed, ints)
    return (mol, ints) if with_ints else mol


def chain_geometry(natoms: int = 200, seed: int = 2):
    """Zig-zag heavy-atom backbone (C/N/O) with one H on every third heavy atom."""
    rng = np.random.default_rng(seed)
    nheavy = (3 * natoms) // 4
    nh = natoms - nheavy
    bond, ch = 1.45, 1.09
    th = math.radians(114.0) / 2.0
    xyz, Z = [], []
    for k in range(nheavy):
        x = k * bond * math.sin(th)
        y = (k % 2) * bond * math.cos(th)
        xyz.append([x, y, 0.0])
        u = rng.random()
        Z.append(6 if u < 0.7 else (7 if u < 0.85 else 8))
    if (sum(Z) + nh) % 2:            # closed shell: even electron count
        k = next(i for i, z in enumerate(Z) if z == 7)
        Z[k] = 6
    hz = 0
    for k in range(0, nheavy, 3):
        if hz >= nh:
            break
        x, y, _ = xyz[k]
        sgn = -1.0 if k % 2 == 0 else 1.0
        xyz.append([x, y + sgn * ch * 0.6, ch * 0.8])
        Z.append(1)
        hz += 1
    k = 1
    while hz < nh:
        x, y, _ = xyz[k]
        xyz.append([x, y, -ch])
        Z.append(1)
        hz += 1
        k += 3
    return np.array(xyz), np.array(Z, dtype=np.int32)


def chain(natoms: int = 200, seed: int = 2, with_ints=False):
    """Config-2 molecule: 200-atom C/N/O/H chain with STO-3G (~800 AOs)."""
    xyz, Z = chain_geometry(natoms, seed)
    mol = Molecule(Z=Z, xyz=_ang(xyz), shells=basis_shells(Z), title=f"C/N/O/H chain {natoms} atoms")
    nelec = int(Z.sum())
    ints = ao_integrals(mol)
    attach_mos(mol, nelec // 2, seed + 100, ints)
    return (mol, ints) if with_ints else mol


def random_molecule(natoms: int, seed: int, with_ints=False):
    """A compact random C/N/O/H cluster (batched / served workloads), STO-3G."""
    rng = np.random.default_rng(seed)
    nheavy = max(1, (2 * natoms) // 3)
    pts = []
    # grow a cluster with >= 1.3 A separation between heavy atoms
    while len(pts) < nheavy:
        if not pts:
            pts.append(np.zeros(3))
            continue
        base = pts[rng.integers(len(pts))]
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        c = base + 1.45 * v
        if min(np.linalg.norm(c - q) for q in pts) > 1.3:
            pts.append(c)
    Z = [6 if rng.random() < 0.7 else (7 if rng.random() < 0.5 else 8) for _ in pts]
    hs = []
    tries = 0
    while len(hs) < natoms - nheavy and tries < 100000:
        tries += 1
        base = pts[rng.integers(len(pts))]
        v = rng.standard_normal(3)
        v /= np.linalg.norm(v)
        c = base + 1.09 * v
        if min(np.linalg.norm(c - q) for q in pts) > 1.0 and all(np.linalg.norm(c - h) > 1.5 for h in hs):
            hs.append(c)
    xyz = np.vstack([np.array(pts), np.array(hs)]) if hs else np.array(pts)
    Z = np.array(Z + [1] * len(hs), dtype=np.int32)
    mol = Molecule(Z=Z, xyz=_ang(xyz), shells=basis_shells(Z), title=f"random cluster {len(Z)} atoms")
    nelec = int(Z.sum())
    ints = ao_integrals(mol)
    attach_mos(mol, nelec // 2, seed + 7, ints)
    return (mol, ints) if with_ints else mol


def open_shell(mol: Molecule, n_alpha: int, n_beta: int, seed: int, ints=None):
    """An unrestricted wavefunction on the molecule's basis: independent
    S-orthonormal alpha and beta MO sets (C = S^-1/2 Q, Q Haar-random), sorted
    uniform orbital energies, occupations 1 / 0 per spin MO.  Returns
    (C [nao, 2 nao], eps, occ, csp) with the alpha MOs first (csp 1, 2)."""
    rng = np.random.default_rng(seed)
    S = (ints if ints is not None else ao_integrals(mol))[0]
    e, U = np.linalg.eigh(S)
    Sm12 = (U / np.sqrt(e)) @ U.T
    n = mol.nao
    Cs, epss, occs = [], [], []
    for ne in (n_alpha, n_beta):
        Cs.append(Sm12 @ haar_orthogonal(n, rng))
        eo = np.sort(rng.uniform(-0.8, -0.2, ne))
        ev = np.sort(rng.uniform(0.0, 0.6, n - ne))
        epss.append(np.concatenate([eo, ev]))
        occs.append(np.concatenate([np.ones(ne), np.zeros(n - ne)]))
    csp = np.concatenate([np.ones(n, dtype=np.int32), np.full(n, 2, dtype=np.int32)])
    return np.hstack(Cs), np.concatenate(epss), np.concatenate(occs), csp

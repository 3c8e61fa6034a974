"""FP64 CPU oracle of std2's sTDA / sTD-DFT path (TEST INFRASTRUCTURE ONLY).

This module is the checker for the CUDA engine.  Only ``tests/``,
``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline leg may import
it; the engine itself never calls it.  It restates, in double precision and
numpy, what ``SUBROUTINE stda`` (``stda.f:53-1606``) does between the AO
integrals and ``tda.dat``, plus the sTD-DFT (``srpapack.f``), the dynamic
polarizability (``linear_response.f:23-192``), the SHG hyperpolarizability
(``linear_response.f:196-700``) and the two-photon absorption
(``linear_response.f:4604-5153``) branches.  The reference keeps
charges, gamma matrices and A in ``real*4``; this oracle keeps everything in
``real*8`` so that it can serve as the FP64 yardstick.  It is pinned against
the reference's golden files (``tests/expected_results/EXCI_TEST*.dat``, the
beta_HRS values of ``BETA_TEST*.txt`` and the excitation energies and 2PA
strengths of ``2PA_TEST*.txt``) by ``tests/test_oracle_golden.py``.

Conscious deviations (also applied by the engine, so both agree bit-for-bit
on the CSF set):

* ``sort_vec`` (``sutda.f:1789``) is called on ``c`` rather than on the active
  copy ``ca`` (``stda.f:333``); here the active MOs *and* their energies are
  sorted together with a stable sort, which is identical for energy-ordered
  input and consistent otherwise.
* The primary-CSF selection sort (``stda.f:651-668``) is not stable for equal
  diagonal energies; here ties are broken by CSF enumeration order (i, a).
"""
from __future__ import annotations

import math
import os
from dataclasses import dataclass, field

import numpy as np
import scipy.linalg as sla

EH2EV_IN = 27.211385050      # stda.f:142 (input conversion)
EH2EV_OUT = 27.21139         # stda.f:1455, print_tdadat
ROT_FAC = -235.7220          # stda.f:1264
NM_FAC = 45.56335            # linear_response.f:85

# atomic chemical hardness eta (Eh), setrep (stda.f:2060-2167)
ETA = np.array([
    0.472592880, 0.922033910, 0.174528880, 0.257007330, 0.339490860,
    0.421954120, 0.504381930, 0.586918630, 0.669313510, 0.751916070,
    0.179641050, 0.221572760, 0.263485780, 0.305396450, 0.347340140,
    0.389247250, 0.431156700, 0.473082690, 0.171054690, 0.202762440,
    0.210073220, 0.217396470, 0.224710390, 0.232015010, 0.239339690,
    0.246656380, 0.253982550, 0.261288630, 0.268594760, 0.275925650,
    0.307629990, 0.339315800, 0.372359850, 0.402735490, 0.434457760,
    0.466117080, 0.155850790, 0.186493240, 0.193562100, 0.200633110,
    0.207705220, 0.214772540, 0.221846140, 0.228918720, 0.235986210,
    0.243056120, 0.250130180, 0.257199370, 0.287847800, 0.318486730,
    0.349124310, 0.379765930, 0.410408080, 0.441057770, 0.050193320,
    0.067625700, 0.085044450, 0.102477360, 0.119911050, 0.137327720,
    0.154762970, 0.172182650, 0.189612880, 0.207047600, 0.224467520,
    0.241896450, 0.259325030, 0.276760940, 0.294182310, 0.311595870,
    0.329022740, 0.345922980, 0.363880480, 0.381305860, 0.398774760,
    0.416142980, 0.433645100, 0.451040140, 0.468489860, 0.485845500,
    0.125267300, 0.142686770, 0.160116150, 0.177558890, 0.194975570,
    0.212407780, 0.072635250, 0.094221580, 0.099202950, 0.104186210,
    0.142356330, 0.163942940, 0.185519410, 0.223701390])

# atomic masses (block.f:24-35) for the MMASS header; index = Z-1
AMS = np.zeros(107)
AMS[:56] = [1.00790, 4.00260, 6.94000, 9.01218, 10.81000, 12.01100, 14.00670,
            15.99940, 18.99840, 20.17900, 22.98977, 24.30500, 26.98154,
            28.08550, 30.97376, 32.06000, 35.45300, 39.94800, 39.09830,
            40.08000, 44.95590, 47.90000, 50.94150, 51.99600, 54.93800,
            55.84700, 58.93320, 58.71000, 63.54600, 65.38000, 69.73500,
            72.59000, 74.92160, 78.96000, 79.90400, 83.80000, 85.46780,
            87.62000, 88.90590, 91.22000, 92.90640, 95.94000, 98.90620,
            101.0700, 102.9055, 106.4000, 107.8680, 112.4100, 114.8200,
            118.6900, 121.7500, 127.6000, 126.9045, 131.3000, 132.9054,
            137.3300]
AMS[71:83] = [178.4900, 180.9479, 183.8500, 186.2070, 190.2000, 192.2200,
              195.0900, 196.9665, 200.5900, 204.3700, 207.2000, 208.9804]
AMS[101] = 1.0079


@dataclass
class Params:
    """Keywords of the sTDA path (``main.f:84-131``, ``stda.f:53-54``)."""
    ax: float = 0.5           # -ax
    e_thr_ev: float = 7.0     # -e  (thre)
    thrp: float = 1e-4        # -p x -> 10**-x
    alpha_k: float = -100.0   # -al (-100: default 1.42+0.48 ax)
    beta_j: float = -100.0    # -be (-100: default 0.20+1.83 ax)
    fthr_ev: float = 1.7976931348623157e308   # -lpt
    triplet: bool = False     # -t
    rpa: bool = False         # -rpa
    velcorr: bool = True      # default for sTDA
    kshift: bool = False      # -xtb / -kshift
    shftmax: float = 0.5
    shftwidth: float = 0.1
    shftsteep: float = 4.0
    shftmax_somo: float = 1.0 # UKS: extra shift of SOMO excitations (main.f:208)


@dataclass
class Result:
    no: int = 0
    nv: int = 0
    occ_idx: np.ndarray = None     # active occupied MO indices (0-based, sorted)
    virt_idx: np.ndarray = None
    eps_act: np.ndarray = None
    nex: int = 0                  # primaries
    nexpt: int = 0                # PT candidates
    new: int = 0                  # PT-selected
    iconf: np.ndarray = None      # (nci, 2) 0-based (i over active occ, a over active virt)
    ed: np.ndarray = None         # (nci,) diagonal after PT lowering
    pt2: np.ndarray = None
    A: np.ndarray = None          # TDA: A ; RPA: (A+B, A-B)
    Apb: np.ndarray = None
    Amb: np.ndarray = None
    omega: np.ndarray = None      # roots in Eh
    X: np.ndarray = None          # (nci, nroot)  TDA X or X (RPA)
    Y: np.ndarray = None
    fL: np.ndarray = None
    fV: np.ndarray = None
    RL: np.ndarray = None
    RV: np.ndarray = None
    alpha0: np.ndarray = None     # packed xx xy yy xz yz zz  (stda.f:1247-1252, x2)
    mu_ia: dict = field(default_factory=dict)
    xmolw: float = 0.0
    extras: dict = field(default_factory=dict)


class OracleError(RuntimeError):
    pass


# ---------------------------------------------------------------- helpers ---

def gamma_matrices(xyz4: np.ndarray, ax: float, alpha_k: float, beta_j: float):
    """gamma^J and gamma^K, Mataga-Nishimoto-Ohno-Klopman form (stda.f:509-532)."""
    Z = np.rint(xyz4[3]).astype(int)
    eta = ETA[Z - 1]
    xyz = xyz4[:3].T
    r = np.sqrt(np.sum((xyz[:, None, :] - xyz[None, :, :]) ** 2, axis=-1))
    etab = 0.5 * (eta[:, None] + eta[None, :])
    xj = etab * ax
    xk = etab
    with np.errstate(divide="ignore"):
        inv_xj = np.where(xj > 0, 1.0 / np.where(xj > 0, xj, 1.0) ** beta_j, np.inf)
    gj = 1.0 / (r ** beta_j + inv_xj) ** (1.0 / beta_j)
    gk = 1.0 / (r ** alpha_k + 1.0 / xk ** alpha_k) ** (1.0 / alpha_k)
    return gj, gk


def default_alpha_beta(p: Params):
    """stda.f:490-500."""
    beta = p.beta_j if p.beta_j >= -99.0 else 0.20 + 1.830 * p.ax
    alpha = p.alpha_k if p.alpha_k >= -99.0 else 1.420 + 0.480 * p.ax
    return alpha, beta


def select_window(eps, occ, ax, thr_eh):
    """Orbital window (stda.f:145-192): returns active occ / virt MO indices."""
    deps = 2.0 * (1.0 + 0.8 * ax) * thr_eh
    occm = occ > 1.990
    virm = occ < 0.010
    omax = eps[occm].max() if occm.any() else -1e42
    vmin = eps[virm].min() if virm.any() else 1e42
    othr = vmin - deps
    vthr = deps + omax
    oidx = np.nonzero(occm & (eps > othr))[0]
    vidx = np.nonzero(virm & (eps < vthr))[0]
    return oidx, vidx


def lowdin_orthogonal_mos(S, Cact):
    """makel (stda.f:1615-1691) + C_low = S^1/2 C (stda.f:436-452)."""
    e, U = np.linalg.eigh(S)
    if (e < 0).any():
        raise OracleError("S^1/2: negative overlap eigenvalue")
    X = (U * np.sqrt(e)) @ U.T
    Clow = X @ Cact
    nrm = np.sum(Clow ** 2, axis=0)
    if (np.abs(nrm - 1.0) > 1e-2).any():
        raise OracleError("internal MO norm error")
    return Clow


def charges(Clow, iaoat, ncent, p_idx, q_idx):
    """lo12pop (stda.f:1727-1744) for MO pairs (p_idx[k], q_idx[k]) -> (ncent, npairs)."""
    prod = Clow[:, p_idx] * Clow[:, q_idx]
    out = np.zeros((ncent, prod.shape[1]))
    np.add.at(out, iaoat, prod)
    return out


def charges_block(Clow, iaoat, ncent, P, Q):
    """lo12pop (stda.f:1727-1744) for every pair of the MO blocks P x Q, pair
    index k = p*len(Q) + q -> (ncent, len(P)*len(Q)); per atom the AO sum is one
    small product C_A[:, P]^T C_A[:, Q] (same sums as ``charges``)."""
    P, Q = np.asarray(P), np.asarray(Q)
    out = np.zeros((ncent, len(P) * len(Q)))
    for A in range(ncent):
        rows = np.nonzero(iaoat == A)[0]
        if len(rows):
            out[A] = (Clow[np.ix_(rows, P)].T @ Clow[np.ix_(rows, Q)]).ravel()
    return out


def mo_ov(mat_ao, C_occ, C_virt):
    """ONETRI (onetri.f:20-55) restricted to the occ-virt block: C_i^T B C_a."""
    return C_occ.T @ mat_ao @ C_virt


# ------------------------------------------------------------- pipeline ---

def stda(xyz4, C, eps, occ, iaoat, S, Lao, Vao, Mao, p: Params, want_A=True, real4=False,
         want_roots=True):
    """Run the sTDA / sTD-DFT excitation path in FP64.

    ``real4=True`` stores what the reference stores in ``real*4`` in single
    precision instead -- charges and gamma matrices (``stda.f:465-532``), the
    gamma.q products (``ssymm``), the couplings, A / A+B / A-B and the
    eigensolves (``ssyevr``, ``sspevd``) -- with the PT sums, the diagonal and
    the properties in double precision as there; it measures how far the
    reference's own arithmetic sits from the FP64 yardstick.

    ``want_A=False`` stops after the PT selection (CSF list and lowered
    diagonal); ``want_roots=False`` with ``rpa`` stops once A+B and A-B are
    built (enough for :func:`dynamic_polarizability`).

    Inputs follow the boundary: ``xyz4`` (4, ncent) Bohr + Z, ``C`` (nao, nmo),
    ``eps``/``occ`` (nmo), ``iaoat`` (nao) 0-based, dense AO matrices ``S``
    (nao, nao) and ``Lao``/``Vao``/``Mao`` (3, nao, nao) with the conventions
    of :mod:`stda_b200.integrals`.
    """
    res = Result()
    ncent = xyz4.shape[1]
    thr = p.e_thr_ev / EH2EV_IN
    fthr = p.fthr_ev / EH2EV_IN if p.fthr_ev < 1.79e308 else np.inf
    Z = np.rint(xyz4[3]).astype(int)
    res.xmolw = float(np.sum(AMS[Z - 1]))

    oidx, vidx = select_window(eps, occ, p.ax, thr)
    no, nv = len(oidx), len(vidx)
    if no == 0 or nv == 0:
        raise OracleError("no CSF, increase energy threshold (-e option)")
    # sort_vec (stda.f:333), stable, applied to active copies
    oo = oidx[np.argsort(eps[oidx], kind="stable")]
    vv = vidx[np.argsort(eps[vidx], kind="stable")]
    res.no, res.nv, res.occ_idx, res.virt_idx = no, nv, oo, vv
    epsi = np.concatenate([eps[oo], eps[vv]])
    res.eps_act = epsi
    Cact = C[:, np.concatenate([oo, vv])]
    Co, Cv = Cact[:, :no], Cact[:, no:]

    # property integrals, occ-virt block (stda.f:351-412)
    mu = {}
    for name, mat in (("L", Lao), ("V", Vao), ("M", Mao)):
        mu[name] = np.stack([mo_ov(mat[d], Co, Cv) for d in range(3)])  # (3,no,nv)
    res.mu_ia = mu
    # occupied-occupied and virtual-virtual length dipoles (the same packed
    # moci x moci transform, stda.f:351-412) for the quadratic response
    res.extras["mu_oo"] = np.stack([Co.T @ Lao[d] @ Co for d in range(3)])
    res.extras["mu_vv"] = np.stack([Cv.T @ Lao[d] @ Cv for d in range(3)])

    Clow = lowdin_orthogonal_mos(S, Cact)
    ak = 0.0 if p.triplet else 2.0
    alpha_k, beta_j = default_alpha_beta(p)
    gj, gk = gamma_matrices(xyz4, p.ax, alpha_k, beta_j)
    fdt = np.float32 if real4 else np.float64
    gj, gk = gj.astype(fdt), gk.astype(fdt)

    io_all, ia_all = np.meshgrid(np.arange(no), np.arange(nv), indexing="ij")
    io_all, ia_all = io_all.ravel(), ia_all.ravel()          # k = i*nv + a
    qii = charges(Clow, iaoat, ncent, np.arange(no), np.arange(no)).astype(fdt)
    qaa = charges(Clow, iaoat, ncent, no + np.arange(nv), no + np.arange(nv)).astype(fdt)
    uci = qaa.T @ (gj @ qii)                                  # (nv, no): (ii|aa)
    qia = charges_block(Clow, iaoat, ncent, np.arange(no), no + np.arange(nv)).astype(fdt)
    pia = gk @ qia
    ek_all = np.einsum("Ak,Ak->k", pia, qia)                  # (ia|ia)
    de_all = (epsi[no + ia_all] - epsi[io_all]) - uci[ia_all, io_all] + ak * ek_all
    if p.kshift:
        sau = p.shftmax * 0.036749320
        wau = p.shftwidth * 0.036749320
        de_all = de_all + sau / (1.0 + (ek_all / wau) ** p.shftsteep)
    prim = de_all <= thr
    cand = (de_all > thr) & (de_all < fthr)
    pk = np.nonzero(prim)[0]
    ck = np.nonzero(cand)[0]
    res.nex, res.nexpt = len(pk), len(ck)
    if len(pk) < 1:
        raise OracleError("no CSF, increase energy threshold (-e option)")
    # energy sort of primaries, ties by enumeration order (stda.f:651-668)
    pk = pk[np.argsort(de_all[pk], kind="stable")]
    ed = de_all[pk].copy()

    # J-type charges for all occ pairs and virt pairs (stda.f:728-763)
    ii, jj = np.meshgrid(np.arange(no), np.arange(no), indexing="ij")
    qoo = charges_block(Clow, iaoat, ncent, np.arange(no), np.arange(no)).reshape(
        ncent, no, no).astype(fdt)
    aa, bb = np.meshgrid(np.arange(nv), np.arange(nv), indexing="ij")
    qvv = charges_block(Clow, iaoat, ncent, no + np.arange(nv), no + np.arange(nv)).reshape(
        ncent, nv, nv).astype(fdt)
    poo = (gj @ qoo.reshape(ncent, -1)).reshape(qoo.shape)

    def coupling(krow, kcol):
        """ak*(ia|jb) - (ij|ab) for CSF index arrays (ravelled i*nv+a)."""
        i1, a1 = io_all[krow], ia_all[krow]
        i2, a2 = io_all[kcol], ia_all[kcol]
        K = pia[:, krow].T @ qia[:, kcol]
        # (ij|ab): gather over the occ/virt boxes actually touched
        ou1, oinv1 = np.unique(i1, return_inverse=True)
        ou2, oinv2 = np.unique(i2, return_inverse=True)
        vu1, vinv1 = np.unique(a1, return_inverse=True)
        vu2, vinv2 = np.unique(a2, return_inverse=True)
        P = poo[:, ou1][:, :, ou2].reshape(ncent, -1)          # (N, o1*o2)
        Q = qvv[:, vu1][:, :, vu2].reshape(ncent, -1)          # (N, v1*v2)
        J4 = (P.T @ Q).reshape(len(ou1), len(ou2), len(vu1), len(vu2))
        J = J4[oinv1[:, None], oinv2[None, :], vinv1[:, None], vinv2[None, :]]
        return ak * K - J

    def exchange(ks):
        """(ib|ja) with gamma^K for CSF pairs u=(i,a), v=(j,b) (rrpamat stda.f:1943-1946)."""
        i1, a1 = io_all[ks], ia_all[ks]
        n = len(ks)
        out = np.empty((n, n), dtype=fdt)
        rb = max(1, int(3e7 // max(1, n * ncent)))
        for r0 in range(0, n, rb):
            r1 = min(n, r0 + rb)
            kib = i1[r0:r1, None] * nv + a1[None, :]
            kja = i1[None, :] * nv + a1[r0:r1, None]
            out[r0:r1] = np.einsum("Auv,Auv->uv", pia[:, kib], qia[:, kja])
        return out

    # PT selection (stda.f:1773-1863)
    pt2 = np.zeros(len(pk))
    incl = np.zeros(len(ck), dtype=bool)
    blk = max(1, int(4e6 // max(1, len(pk))))
    for s0 in range(0, len(ck), blk):
        kk = ck[s0:s0 + blk]
        amat = coupling(kk, pk)                                  # (nk, nex)
        pt = amat ** 2 / (de_all[kk][:, None] - ed[None, :] + 1e-10)
        pert = pt.sum(axis=1)
        sel = pert > p.thrp
        incl[s0:s0 + blk] = sel
        pt2 += pt[~sel].sum(axis=0)
    newk = ck[incl]
    res.new = len(newk)
    res.pt2 = pt2
    ed = np.concatenate([ed - pt2, de_all[newk]])
    allk = np.concatenate([pk, newk])
    nci = len(allk)
    res.iconf = np.stack([io_all[allk], ia_all[allk]], axis=1)
    res.ed = ed
    res.extras.update(de_all=de_all, ek_all=ek_all, pk=pk, ck=ck, allk=allk,
                      pair_tensors=(pia, qia, poo, qvv))

    mL = mu["L"][:, io_all[allk], ia_all[allk]]              # (3, nci)
    mV = mu["V"][:, io_all[allk], ia_all[allk]]
    mM = mu["M"][:, io_all[allk], ia_all[allk]]

    if not want_A:
        return res

    # A matrix (rtdamat stda.f:2010-2056), built in row blocks to bound memory
    A = np.empty((nci, nci), dtype=fdt)
    rb = max(1, int(2e7 // max(1, nci)))
    for r0 in range(0, nci, rb):
        A[r0:r0 + rb] = coupling(allk[r0:r0 + rb], allk)
    np.fill_diagonal(A, ed)

    if p.rpa:
        # exchange-type (ib|ja) with gamma^K (rrpamat stda.f:1930-1963)
        Kx = exchange(allk)
        Kd = ek_all[allk]
        Kov = pia[:, allk].T @ qia[:, allk]
        Apb = 2.0 * ak * Kov - p.ax * Kx - (ak * Kov - A)       # 2ak(ia|jb) - ax(ib|ja) - (ij|ab)
        Amb = p.ax * Kx - (ak * Kov - A)                         # ax(ib|ja) - (ij|ab)
        np.fill_diagonal(Apb, ed - p.ax * Kd + ak * Kd)
        np.fill_diagonal(Amb, ed - ak * Kd + p.ax * Kd)
        if abs(p.ax) < 1e-6:
            Amb = np.diag(ed - ak * Kd).astype(fdt)
        res.Apb, res.Amb = Apb, Amb
        if not want_roots:
            # A+B, A-B only (what lresp needs, linear_response.f:23-192)
            return res
        # srpapack (srpapack.f:32-197): M = (A-B)^1/2 (A+B) (A-B)^1/2
        e, U = np.linalg.eigh(Amb)
        if e[0] < 0:
            raise OracleError("matrix power impossible")
        Ambh = (U * np.sqrt(e)) @ U.T
        Mmat = Ambh @ Apb @ Ambh
        w, Zv = sla.eigh(Mmat, subset_by_value=(0.0, thr * thr))
        if len(w) < 1:
            raise OracleError("RPA diag failed")
        om = np.sqrt(w)
        XpY = (Ambh @ Zv) / np.sqrt(om)
        XmY = (Apb @ XpY) / om
        X = 0.5 * (XpY + XmY)
        Y = XpY - X
        res.omega, res.X, res.Y = om, X, Y
        res.extras["Ambh"], res.extras["Z_rpa"] = Ambh, Zv
        uu, pp = XpY, XmY
    else:
        res.A = A
        w, Xv = sla.eigh(A, subset_by_value=(0.0, thr))
        if len(w) < 1:
            raise OracleError("internal error in diag")
        res.omega, res.X = w, Xv
        uu = pp = Xv

    # properties (stda.f:1207-1289)
    sak = math.sqrt(ak)
    om = res.omega
    ef = 1.0 / (om + 1e-8)
    tl = sak * (mL @ uu)          # (3, nroot)
    tv = sak * (mV @ pp)
    tm = sak * (mM @ pp)
    res.fL = om * (2.0 / 3.0) * np.sum(tl * tl, axis=0)
    res.fV = ef * (2.0 / 3.0) * np.sum(tv * tv, axis=0)
    res.RL = ROT_FAC * np.sum(tl * tm, axis=0)
    res.RV = ROT_FAC * np.sum(tv * tm, axis=0) * ef
    a = np.array([np.sum(tl[0] * tl[0] * ef), np.sum(tl[0] * tl[1] * ef), np.sum(tl[1] * tl[1] * ef),
                  np.sum(tl[0] * tl[2] * ef), np.sum(tl[1] * tl[2] * ef), np.sum(tl[2] * tl[2] * ef)])
    res.alpha0 = 2.0 * a

    if (not p.rpa) and p.velcorr:
        # rtdacorr (apbtrafo.f:580-643) + apbtrafo (apbtrafo.f:23-300)
        Kx = exchange(allk)
        Kov = pia[:, allk].T @ qia[:, allk]
        Bh = 0.5 * ak * Kov - 0.5 * p.ax * Kx
        np.fill_diagonal(Bh, 0.5 * (ak * np.diag(Kov) - p.ax * np.diag(Kov)))
        Xn = (Bh @ res.X) * ef[None, :]
        xl = mL @ res.X
        xv = mV @ res.X
        xm = mM @ res.X
        xv2 = mV @ Xn
        xm2 = mM @ Xn
        hilf = 1.0 - np.exp(-150.0 * om * om)
        efmod = 1.0 / (om ** hilf + 1e-8)
        p23 = ak * 2.0 / 3.0
        res.fL = np.sum(xl * xl, axis=0) * p23 * om
        res.fV = p23 * ef * np.sum(xv * xv, axis=0)
        res.RL = ROT_FAC * np.sum(xl * xm, axis=0) * ak
        res.RV = ROT_FAC * np.sum(xv * xm + xv2 * xm + xv * xm2, axis=0) * ak * efmod
        res.extras["Bhalf"] = Bh
    return res


def tda_dat_text(res: Result, p: Params) -> str:
    """tda.dat as written by apbtrafo (velocity-corrected sTDA, apbtrafo.f:100-243)
    or print_tdadat (stda.f:2235-2265) otherwise."""
    velo = (not p.rpa) and p.velcorr
    thr = p.e_thr_ev / EH2EV_IN
    lines = [" NM", " VELO" if velo else " UV", " MMASS", f"   {res.xmolw:.15f}     ",
             " LFAKTOR", "  0.5", " RFAKTOR", "  1.0", " WIDTH", "  0.20", " SHIFT", "  0.00", " DATXY"]
    for i, om in enumerate(res.omega):
        if (not velo) and om > thr:
            continue
        lines.append("%4d%10.4f%13.6f%13.6f%13.6f%13.6f" % (
            i + 1, om * EH2EV_OUT, res.fL[i], res.fV[i], res.RL[i], res.RV[i]))
    return "\n".join(lines) + "\n"


def dynamic_polarizability(res: Result, omegas_eh) -> np.ndarray:
    """lresp (linear_response.f:23-192): alpha(omega) for each omega (Eh).

    Solves [(A+B) - w^2 (A-B)^-1] (X+Y) = -2 mu for the three Cartesian
    right-hand sides and returns alpha[w, x, y] = -2 sum mu_x (X+Y)_y.
    Requires a result computed with ``Params(rpa=True)``.
    """
    if res.Apb is None:
        raise OracleError("dynamic polarizability needs the A+B / A-B matrices (rpa=True)")
    nv = res.nv
    allk = res.extras["allk"]
    i1, a1 = allk // nv, allk % nv
    mL = res.mu_ia["L"][:, i1, a1]                    # (3, nci)
    # the solves run in the matrices' precision (real*4 ssptrf / ssptrs in the
    # reference, FP64 here unless the result came from the real*4 mode); the
    # sums over CSFs are real*8 in both
    dt = res.Apb.dtype
    rhs = (-2.0 * mL.T).astype(dt)
    inv_amb = np.linalg.inv(res.Amb)
    out = []
    for w in omegas_eh:
        Mw = res.Apb - dt.type(w * w) * inv_amb
        XpY = np.linalg.solve(Mw, rhs).astype(np.float64)
        out.append(-2.0 * mL @ XpY)
    return np.array(out)


def _xy_vectors(res: Result, w: float, inv_amb, rhs):
    """X and Y of the linear response at frequency w (Eh, may be negative):
    X+Y from [(A+B) - w^2 (A-B)^-1](X+Y) = rhs, X-Y = w (A-B)^-1 (X+Y)
    (linear_response.f:312-327, 371-396)."""
    XpY = np.linalg.solve(res.Apb - (w * w) * inv_amb, rhs)
    XmY = w * (inv_amb @ XpY)
    return 0.5 * (XpY + XmY), 0.5 * (XpY - XmY)


def _hrs_invariants(b):
    """<beta^2_ZZZ>, <beta^2_XZZ> of the hyper-Rayleigh orientational average
    (HRS, linear_response.f:1489-1662); i, j, k run over distinct axes."""
    ax3 = range(3)
    pairs = [(i, j) for i in ax3 for j in ax3 if i != j]
    trip = [(i, j, k) for i in ax3 for j in ax3 for k in ax3 if len({i, j, k}) == 3]
    s_iii = sum(b[i, i, i] ** 2 for i in ax3)
    s_iij = sum(b[i, i, j] ** 2 for i, j in pairs)
    s_jii = sum(b[j, i, i] ** 2 for i, j in pairs)
    s_ijj = sum(b[i, j, j] ** 2 for i, j in pairs)
    s_ijk = sum(b[i, j, k] ** 2 for i, j, k in trip)
    iii_ijj = sum(b[i, i, i] * b[i, j, j] for i, j in pairs)
    jii_iij = sum(b[j, i, i] * b[i, i, j] for i, j in pairs)
    iii_jji = sum(b[i, i, i] * b[j, j, i] for i, j in pairs)
    iij_jii = sum(b[i, i, j] * b[j, i, i] for i, j in pairs)
    iij_jkk = sum(b[i, i, j] * b[j, k, k] for i, j, k in trip)
    jii_jkk = sum(b[j, i, i] * b[j, k, k] for i, j, k in trip)
    iij_kkj = sum(b[i, i, j] * b[k, k, j] for i, j, k in trip)
    ijk_jik = sum(b[i, j, k] * b[j, i, k] for i, j, k in trip)
    ijj_ikk = sum(b[i, j, j] * b[i, k, k] for i, j, k in trip)
    iik_jjk = sum(b[i, i, k] * b[j, j, k] for i, j, k in trip)
    zzz = (s_iii / 7 + 4 * s_iij / 35 + s_jii / 35 + 2 * s_ijk / 105 + 2 * iii_ijj / 35
           + 4 * jii_iij / 35 + 4 * iii_jji / 35 + 4 * iij_jkk / 105 + jii_jkk / 105
           + 4 * iij_kkj / 105 + 4 * ijk_jik / 105)
    xzz = (s_iii / 35 + 4 * iii_ijj / 105 - 2 * iii_jji / 35 + 8 * s_iij / 105
           - 2 * iij_jkk / 105 + 2 * s_ijk / 35 - 2 * ijk_jik / 105 + 3 * s_ijj / 35
           - 2 * iij_jii / 35 + ijj_ikk / 35 - 2 * iik_jjk / 105)
    return zzz, xzz


def _mu_csf(res: Result):
    """Length dipoles of the selected CSFs, (3, nci)."""
    allk = res.extras["allk"]
    return res.mu_ia["L"][:, allk // res.nv, allk % res.nv]


def _dipole_couplings(res: Result):
    """Per axis d the nci x nci matrix that couples CSF p to CSF q in the
    quadratic-response sums (List_A / List_B, linear_response.f:1089-1167):
    -mu_ij when p = (i a), q = (j a) share their virtual, minus -mu_ab when
    p = (i a), q = (i b) share their occupied, so that X M Y = A - B."""
    allk = res.extras["allk"]
    io, iv = allk // res.nv, allk % res.nv
    same_v = iv[:, None] == iv[None, :]
    same_o = io[:, None] == io[None, :]
    M = []
    for d in range(3):
        moo = res.extras["mu_oo"][d][io[:, None], io[None, :]]
        mvv = res.extras["mu_vv"][d][iv[:, None], iv[None, :]]
        M.append(np.where(same_v, -moo, 0.0) - np.where(same_o, -mvv, 0.0))
    return M


def shg_hyperpolarizability(res: Result, wavelengths_nm):
    """lresp1 (linear_response.f:196-700; beta_resp_fast :911-1087, List_A /
    List_B :1089-1167, A_beta_fast / B_beta_fast :1170-1226, HRS :1489-1662):
    the second-harmonic first hyperpolarizability beta(-2w; w, w) of sTD-DFT
    and its hyper-Rayleigh value beta_HRS, at w = 0 and w = 45.56335 / lambda.

    The linear responses to -2 mu at +w and at -2w give X, Y per axis.  With
    the CSF pairs (i a), (j a) that share their virtual (coupled through
    mu_ij) and (i a), (i b) that share their occupied (coupled through mu_ab),
    beta = A - B (no derivative of the XC kernel), each of A and B summed over
    the six assignments of (x, y, z) to the -2w X vector, the dipole and the
    w Y vector that lresp1 lists.  Every component is computed directly (the
    reference copies the permutation-equivalent ones, which the sum makes
    equal).  Returns (w in eV as printed, beta[nw, 3, 3, 3], beta_HRS[nw]).
    """
    if res.Apb is None:
        raise OracleError("the hyperpolarizability needs A+B / A-B (rpa=True)")
    rhs = -2.0 * _mu_csf(res).T                                # (nci, 3)
    inv_amb = np.linalg.inv(res.Amb)
    M = _dipole_couplings(res)
    freqs = [0.0] + [NM_FAC / float(lam) for lam in wavelengths_nm]
    betas, hrs = [], []
    for f in freqs:
        X1, Y1 = _xy_vectors(res, f, inv_amb, rhs)           # +w
        X2, Y2 = _xy_vectors(res, -2.0 * f, inv_amb, rhs)    # -2w
        Xs, Ys = {1: X1, 2: X2}, {1: Y1, 2: Y2}

        def term(x, wx, y, z, wz):
            return Xs[wx][:, x] @ M[y] @ Ys[wz][:, z]

        b = np.zeros((3, 3, 3))
        for i in range(3):
            for j in range(3):
                for k in range(3):
                    b[i, j, k] = (term(i, 2, j, k, 1) + term(i, 2, k, j, 1)
                                  + term(j, 1, k, i, 2) + term(j, 1, i, k, 1)
                                  + term(k, 1, i, j, 1) + term(k, 1, j, i, 2))
        zzz, xzz = _hrs_invariants(b)
        betas.append(b)
        hrs.append(math.sqrt(zzz + xzz))
    return np.array(freqs) * EH2EV_OUT, np.array(betas), np.array(hrs)


def two_photon_absorption(res: Result, ntrans: int):
    """lresp_2PA_SP (linear_response.f:4604-4938; TPA_resp_fast_SP :4940-5025,
    A/B_2PA_*_fast_SP :5027-5153): two-photon absorption of the lowest
    ``ntrans`` sTD-DFT states in the single-photon-resonance form.

    For state n (energy w_n) the response to -mu at w = -w_n / 2 gives X, Y per
    axis; the two-photon tensor is
      sigma_xy = -1/2 [X_x M_y Yn + X_y M_x Yn + Xn M_x Y_y + Xn M_y Y_x]
    with the CSF couplings M of the quadratic response, and F, G, H (each / 30)
    give delta_par = 2F+2G+2H, delta_perp = -F+4G-H, delta_circ = -2F+3G+3H
    and rho = delta_par / delta_perp.

    Under -2PA the reference's srpapack skips the halving of the packed
    diagonals of (A-B)^1/2 and A+B before its packed products
    (srpapack.f:99-106, 116-133), so its state vectors Xn, Yn carry each
    diagonal twice; this restatement does the same so that it reproduces the
    2PA goldens.  (The excitation energies, and every other consumer of the
    state vectors, use the regular vectors.)  Returns rows
    (n, w_n in eV, delta_par, delta_perp, delta_circ, rho) as in ``2PA-abs``.
    """
    if res.Apb is None or "Z_rpa" not in res.extras:
        raise OracleError("two-photon absorption needs the sTD-DFT states (rpa=True)")
    om = res.omega
    if ntrans > len(om):
        raise OracleError("number of 2PA excitations too large!")
    Sh, Z = res.extras["Ambh"], res.extras["Z_rpa"]
    Sq = Sh + np.diag(np.diag(Sh))
    Pq = res.Apb + np.diag(np.diag(res.Apb))
    XpYn = (Sq @ Z) / np.sqrt(om)
    XmYn = (Pq @ XpYn) / om
    Xn = 0.5 * (XpYn + XmYn)
    Yn = XpYn - Xn
    inv_amb = np.linalg.inv(res.Amb)
    rhs = -_mu_csf(res).T
    M = _dipole_couplings(res)
    rows = []
    for n in range(ntrans):
        X, Y = _xy_vectors(res, -0.5 * om[n], inv_amb, rhs)
        sg = np.empty((3, 3))
        for x in range(3):
            for y in range(3):
                sg[x, y] = -0.5 * (X[:, x] @ M[y] @ Yn[:, n] + X[:, y] @ M[x] @ Yn[:, n]
                                   + Xn[:, n] @ M[x] @ Y[:, y] + Xn[:, n] @ M[y] @ Y[:, x])
        F = np.trace(sg) ** 2 / 30.0
        G = float(np.sum(sg * sg)) / 30.0
        H = float(np.sum(sg * sg.T)) / 30.0
        par, perp = 2 * F + 2 * G + 2 * H, -F + 4 * G - H
        rows.append([n + 1, om[n] * EH2EV_OUT, par, perp, -2 * F + 3 * G + 3 * H, par / perp])
    return np.array(rows)


def read_tda_dat(text: str):
    """Parse the DATXY rows of a tda.dat text into an (n, 6) array."""
    rows = []
    on = False
    for ln in text.splitlines():
        if "DATXY" in ln:
            on = True
            continue
        if on and ln.strip():
            rows.append([float(t) for t in ln.split()])
    return np.array(rows)


_HERE = os.path.dirname(os.path.abspath(__file__))
PAIRLOOPS_SRC = os.path.join(_HERE, "pairloops.c")
PAIRLOOPS_LIB = os.path.join(_HERE, "libpairloops.so")
_pairloops_lib = None


def build_pairloops(force: bool = False) -> str:
    """Compile ``pairloops.c`` (the reference's PT-selection and A-build loops
    in C with OpenMP) next to it with gcc; returns the library path."""
    import subprocess
    stale = (not os.path.exists(PAIRLOOPS_LIB)
             or os.path.getmtime(PAIRLOOPS_SRC) > os.path.getmtime(PAIRLOOPS_LIB))
    if force or stale:
        tmp = PAIRLOOPS_LIB + ".tmp"
        subprocess.run(["gcc", "-O3", "-fopenmp", "-fPIC", "-shared", "-o", tmp, PAIRLOOPS_SRC],
                       check=True, capture_output=True)
        os.replace(tmp, PAIRLOOPS_LIB)
    return PAIRLOOPS_LIB


def pairloops():
    """ctypes handle of the C pair loops, built on first use when missing."""
    global _pairloops_lib
    if _pairloops_lib is None:
        import ctypes as C
        lib = C.CDLL(build_pairloops())
        fp, ip, dp = C.POINTER(C.c_float), C.POINTER(C.c_int), C.POINTER(C.c_double)
        lib.pairloops_ptselect.argtypes = [C.c_int, C.c_int, fp, fp, fp, fp, C.c_int, ip, ip, dp,
                                           C.c_int, ip, ip, dp, C.c_double, C.c_double,
                                           C.POINTER(C.c_ubyte), dp]
        lib.pairloops_ptselect.restype = C.c_int
        lib.pairloops_rtdamat_rows.argtypes = [C.c_int, C.c_int, fp, fp, fp, fp, C.c_int, ip, ip,
                                               dp, C.c_double, C.c_int, C.c_int, fp]
        lib.pairloops_rtdamat_rows.restype = None
        _pairloops_lib = lib
    return _pairloops_lib


class PairTensors32:
    """The reference's real*4 pair tensors in the layout of ``pairloops.c``:
    one contiguous column of N atoms per ia pair (p_ia, q_ia) and per packed
    occupied / virtual pair (p_ij, q_ab, ``lin`` order)."""

    def __init__(self, pia, qia, poo, qvv):
        no, nv = poo.shape[1], qvv.shape[1]
        f4 = np.float32
        self.N, self.nv = pia.shape[0], nv
        self.pia = np.ascontiguousarray(pia.T, dtype=f4)
        self.qia = np.ascontiguousarray(qia.T, dtype=f4)
        hi, lo = np.tril_indices(no)
        self.pij = np.ascontiguousarray(poo[:, hi, lo].T, dtype=f4)
        hi, lo = np.tril_indices(nv)
        self.qab = np.ascontiguousarray(qvv[:, hi, lo].T, dtype=f4)

    def _ptrs(self):
        import ctypes as C
        fp = C.POINTER(C.c_float)
        return [a.ctypes.data_as(fp) for a in (self.pia, self.qia, self.pij, self.qab)]

    def ptselect(self, kio, kiv, edpt, jo, jv, ed, ak, thrp):
        """ptselect's loop (stda.f:1773-1863) for the given candidates and
        primaries: (selected flags, pt2 of the unselected)."""
        import ctypes as C
        ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
        kio, kiv, jo, jv = (np.ascontiguousarray(x, dtype=np.int32) for x in (kio, kiv, jo, jv))
        edpt, ed = (np.ascontiguousarray(x, dtype=np.float64) for x in (edpt, ed))
        incl = np.zeros(len(kio), dtype=np.uint8)
        pt2 = np.zeros(len(jo))
        pairloops().pairloops_ptselect(
            self.N, self.nv, *self._ptrs(), len(kio), kio.ctypes.data_as(ip),
            kiv.ctypes.data_as(ip), edpt.ctypes.data_as(dp), len(jo), jo.ctypes.data_as(ip),
            jv.ctypes.data_as(ip), ed.ctypes.data_as(dp), float(ak), float(thrp),
            incl.ctypes.data_as(C.POINTER(C.c_ubyte)), pt2.ctypes.data_as(dp))
        return incl.astype(bool), pt2

    def rtdamat_rows(self, io, iv, ed, ak, r0, r1):
        """Rows r0..r1-1 of rtdamat's lower triangle (stda.f:2010-2056)."""
        import ctypes as C
        ip, dp = C.POINTER(C.c_int), C.POINTER(C.c_double)
        io, iv = (np.ascontiguousarray(x, dtype=np.int32) for x in (io, iv))
        ed = np.ascontiguousarray(ed, dtype=np.float64)
        rows = np.zeros((r1 - r0, len(io)), dtype=np.float32)
        pairloops().pairloops_rtdamat_rows(
            self.N, self.nv, *self._ptrs(), len(io), io.ctypes.data_as(ip), iv.ctypes.data_as(ip),
            ed.ctypes.data_as(dp), float(ak), r0, r1, rows.ctypes.data_as(C.POINTER(C.c_float)))
        return rows


def stda_timed(xyz4, C, eps, occ, iaoat, S, Lao, Vao, Mao, p: Params, budget_s=15.0):
    """Wall-clock estimate of one full FP64 CPU solve from a bounded sample.

    Phases that are cheap run in full (window, MO integrals, S^1/2, charges,
    gamma, screen).  The PT selection and the A build run the reference's own
    loops (``pairloops.c``: two real*4 dots of length N per CSF pair, OpenMP
    over candidates / rows).  The PT selection runs on blocks of 64 consecutive
    candidates spread evenly over the candidate list until about half the
    budget is used and is scaled linearly to all candidates (also the estimate
    of the selected count: the selection rate varies along the list, and
    blocks of 288 gave a 9x undercount on the C384H48 flake where blocks of 64
    came within 7 %); the A build is timed on the last rows of the primary
    block and scaled by CSF pairs to nci (nci-1) / 2; the dense diagonalisation (ssyevr('V','V') in real*4
    in the reference) is timed as the same call, scipy's ``evr`` driver in
    single precision for the lowest nex/nci fraction of a min(nci, 4000)-sized
    matrix, and scaled as n^3.  Used only as the reported CPU baseline, never
    as a result.
    """
    st = _cpu_setup(xyz4, C, eps, occ, iaoat, S, Lao, Vao, Mao, p)
    return _timed_sample(st, p, budget_s)


def _cpu_setup(xyz4, C, eps, occ, iaoat, S, Lao, Vao, Mao, p: Params):
    """The phases of the CPU restatement that run in full in both the sampled
    estimate and the complete timed solve: window, MO integrals, S^1/2,
    charges, gamma, gamma.q and the diagonal screen (numpy, FP64)."""
    import time
    t_all = time.perf_counter()
    thr = p.e_thr_ev / EH2EV_IN
    oidx, vidx = select_window(eps, occ, p.ax, thr)
    no, nv = len(oidx), len(vidx)
    Cact = C[:, np.concatenate([oidx, vidx])]
    Co, Cv = Cact[:, :no], Cact[:, no:]
    for mat in (Lao, Vao, Mao):
        for d in range(3):
            mo_ov(mat[d], Co, Cv)
    Clow = lowdin_orthogonal_mos(S, Cact)
    epsi = np.concatenate([eps[oidx], eps[vidx]])
    ak = 0.0 if p.triplet else 2.0
    alpha_k, beta_j = default_alpha_beta(p)
    gj, gk = gamma_matrices(xyz4, p.ax, alpha_k, beta_j)
    ncent = xyz4.shape[1]
    io_all, ia_all = np.meshgrid(np.arange(no), np.arange(nv), indexing="ij")
    io_all, ia_all = io_all.ravel(), ia_all.ravel()
    qii = charges(Clow, iaoat, ncent, np.arange(no), np.arange(no))
    qaa = charges(Clow, iaoat, ncent, no + np.arange(nv), no + np.arange(nv))
    uci = qaa.T @ (gj @ qii)
    qia = charges_block(Clow, iaoat, ncent, np.arange(no), no + np.arange(nv))
    pia = gk @ qia
    ek_all = np.einsum("Ak,Ak->k", pia, qia)
    de_all = (epsi[no + ia_all] - epsi[io_all]) - uci[ia_all, io_all] + ak * ek_all
    pk = np.nonzero(de_all <= thr)[0]
    ck = np.nonzero(de_all > thr)[0]
    pk = pk[np.argsort(de_all[pk], kind="stable")]
    ed = de_all[pk]
    ii, jj = np.meshgrid(np.arange(no), np.arange(no), indexing="ij")
    qoo = charges_block(Clow, iaoat, ncent, np.arange(no), np.arange(no)).reshape(ncent, no, no)
    aa, bb = np.meshgrid(np.arange(nv), np.arange(nv), indexing="ij")
    qvv = charges_block(Clow, iaoat, ncent, no + np.arange(nv), no + np.arange(nv)).reshape(ncent, nv, nv)
    poo = (gj @ qoo.reshape(ncent, -1)).reshape(qoo.shape)
    t_setup = time.perf_counter() - t_all
    return dict(thr=thr, ak=ak, ncent=ncent, io_all=io_all, ia_all=ia_all, pia=pia, qia=qia,
                poo=poo, qvv=qvv, de_all=de_all, pk=pk, ck=ck, ed=ed, t_setup=t_setup)


def _pair_loops(st):
    """The reference's own pair loops (ptselect, rtdamat: two real*4 dots of
    length N per CSF pair, OpenMP) in C when gcc can build them, else None."""
    try:
        pt32 = PairTensors32(st["pia"], st["qia"], st["poo"], st["qvv"])
        pairloops()
        return pt32
    except Exception:
        return None


def stda_full_timed(xyz4, C, eps, occ, iaoat, S, Lao, Vao, Mao, p: Params):
    """One complete CPU solve with the pieces stda_timed samples, timed phase
    by phase: the full PT selection and the full A build with the reference's
    pair loops (pairloops.c), and the real*4 evr eigensolve of the roots in
    (0, E_thr] of that A.  Used to check the sampled estimate at a size where
    the complete solve finishes in seconds; never a result."""
    import time
    st = _cpu_setup(xyz4, C, eps, occ, iaoat, S, Lao, Vao, Mao, p)
    pt32 = _pair_loops(st)
    if pt32 is None:
        raise OracleError("the complete timed solve needs the C pair loops (gcc)")
    io_all, ia_all, de_all = st["io_all"], st["ia_all"], st["de_all"]
    pk, ck, ed, ak = st["pk"], st["ck"], st["ed"], st["ak"]
    t0 = time.perf_counter()
    incl, pt2 = pt32.ptselect(io_all[ck], ia_all[ck], de_all[ck], io_all[pk], ia_all[pk], ed, ak,
                              p.thrp)
    t_pt = time.perf_counter() - t0
    allk = np.concatenate([pk, ck[incl]])
    ed_all = np.concatenate([ed - pt2, de_all[ck[incl]]])
    nci = len(allk)
    t0 = time.perf_counter()
    A = pt32.rtdamat_rows(io_all[allk], ia_all[allk], ed_all, ak, 0, nci)
    t_a = time.perf_counter() - t0
    t0 = time.perf_counter()
    sla.eigh(A, lower=True, subset_by_value=(0.0, st["thr"]), driver="evr",
             overwrite_a=True, check_finite=False)
    t_eig = time.perf_counter() - t0
    return dict(total_s=st["t_setup"] + t_pt + t_a + t_eig, setup_s=st["t_setup"], pt_s=t_pt,
                a_s=t_a, eig_s=t_eig, nci=nci)


def _timed_sample(st, p: Params, budget_s):
    """The sampled phases of stda_timed (see there)."""
    import os
    import time
    thr, ak, ncent = st["thr"], st["ak"], st["ncent"]
    io_all, ia_all, pia, qia, poo, qvv = (st[k] for k in ("io_all", "ia_all", "pia", "qia",
                                                          "poo", "qvv"))
    de_all, pk, ck, ed, t_setup = st["de_all"], st["pk"], st["ck"], st["ed"], st["t_setup"]

    def coupling(krow, kcol):
        i1, a1 = io_all[krow], ia_all[krow]
        i2, a2 = io_all[kcol], ia_all[kcol]
        K = pia[:, krow].T @ qia[:, kcol]
        ou1, oinv1 = np.unique(i1, return_inverse=True)
        ou2, oinv2 = np.unique(i2, return_inverse=True)
        vu1, vinv1 = np.unique(a1, return_inverse=True)
        vu2, vinv2 = np.unique(a2, return_inverse=True)
        P = poo[:, ou1][:, :, ou2].reshape(ncent, -1)
        Q = qvv[:, vu1][:, :, vu2].reshape(ncent, -1)
        J4 = (P.T @ Q).reshape(len(ou1), len(ou2), len(vu1), len(vu2))
        return ak * K - J4[oinv1[:, None], oinv2[None, :], vinv1[:, None], vinv2[None, :]]

    # The reference's own loops (ptselect, rtdamat: two real*4 dots of length
    # N per CSF pair, OpenMP) in C when gcc can build them; otherwise the
    # numpy form above, which the sample text then names
    pt32 = _pair_loops(st)
    loops = ("C restatement of ptselect / rtdamat (real*4 dots, OpenMP)" if pt32 is not None
             else "numpy GEMM form of ptselect / rtdamat")

    # PT selection on a sample of candidate blocks spread evenly over the
    # candidate list (the selection rate varies along it), scaled linearly
    t0 = time.perf_counter()
    done, nsel = 0, 0
    blk, group = 64, 8
    nblk_all = max(1, -(-len(ck) // blk))
    order = np.argsort((np.arange(nblk_all) * 0.6180339887) % 1.0, kind="stable")
    for g0 in range(0, len(order), group):
        if time.perf_counter() - t0 >= 0.5 * budget_s:
            break
        kk = np.concatenate([ck[b * blk:(b + 1) * blk] for b in order[g0:g0 + group]])
        if pt32 is not None:
            incl, _ = pt32.ptselect(io_all[kk], ia_all[kk], de_all[kk], io_all[pk], ia_all[pk],
                                    ed, ak, p.thrp)
            nsel += int(incl.sum())
        else:
            amat = coupling(kk, pk)
            pert = (amat ** 2 / (de_all[kk][:, None] - ed[None, :] + 1e-10)).sum(axis=1)
            nsel += int((pert > p.thrp).sum())
        done += len(kk)
    t_pt = (time.perf_counter() - t0) * len(ck) / max(1, done)
    nci = len(pk) + int(round(nsel * len(ck) / max(1, done)))
    # A build: rtdamat fills the lower triangle, nci (nci-1) / 2 pairs; time the
    # last rows of the primary block and scale by pairs
    t0 = time.perf_counter()
    r1 = len(pk)
    r0 = max(0, r1 - 256)
    if pt32 is not None:
        pt32.rtdamat_rows(io_all[pk], ia_all[pk], ed, ak, r0, r1)
        pairs = (r0 + r1 - 1) * (r1 - r0) / 2.0
    else:
        coupling(pk[r0:r1], pk)
        pairs = float(r1 - r0) * r1
    rows = pk[r0:r1]
    t_a = (time.perf_counter() - t0) * (nci * (nci - 1) / 2.0) / max(1.0, pairs)
    # dense diagonalisation, the roots below E_thr (about nex of them), scaled as n^3
    # (sizes below ~3000 run at poor parallel efficiency and overstate the
    # n^3 extrapolation by ~2x: 6467 s from 1500 against 2864 s from 4500 for
    # the C384H48 flake on 8 cores)
    n_s = min(nci, 4000)
    k_s = max(1, min(n_s, int(round(n_s * len(pk) / max(1, nci)))))
    rng = np.random.default_rng(0)
    Mx = rng.standard_normal((n_s, n_s)).astype(np.float32)
    Mx = Mx + Mx.T
    t0 = time.perf_counter()
    sla.eigh(Mx, subset_by_index=[0, k_s - 1], driver="evr")
    t_eig = (time.perf_counter() - t0) * (nci / n_s) ** 3
    est = t_setup + t_pt + t_a + t_eig
    threads = int(os.environ.get("OMP_NUM_THREADS", os.cpu_count() or 1))
    sample = (f"{loops}; full window/S^1/2/charges/screen ({t_setup:.1f}s); PT on {done} of {len(ck)} "
              f"candidates (blocks of {blk} spread evenly) x {len(pk)} primaries scaled "
              f"linearly ({t_pt:.1f}s est.); A build "
              f"{len(rows)} rows scaled to nci={nci} ({t_a:.1f}s est.); real*4 evr eigh, "
              f"lowest {k_s} of {n_s}, scaled to nci^3 ({t_eig:.1f}s est.)")
    return dict(est_total_s=est, setup_s=t_setup, pt_s=t_pt, a_s=t_a, eig_s=t_eig, nci=nci,
                threads=threads, sample=sample)


def dominant_csfs(res: Result):
    """The three dominant CSFs of each root as the reference picks them for
    its state table (stda.f:1222-1358): over the CSFs in order, with
    u = X + Y, p = X - Y (sTD-DFT) or u = p = X (TDA), the first is the last
    CSF where |u p| exceeded the running value umax (which then becomes u p,
    signed), the second and third where u p exceeded it (umax reset to -1,
    earlier picks skipped).  Returns (value, i, a) arrays of shape (nroot, 3):
    value = the TDA coefficient or X^2 - Y^2; i, a = the occupied and virtual
    MO of the CSF, 1-based, virtual numbered after the no occupied MOs."""
    X = res.X
    Y = res.Y if res.Y is not None else None
    nci, nroot = X.shape
    val = np.zeros((nroot, 3))
    oi = np.zeros((nroot, 3), dtype=int)
    oa = np.zeros((nroot, 3), dtype=int)
    for r in range(nroot):
        x = X[:, r]
        y = Y[:, r] if Y is not None else np.zeros(nci)
        up = (x + y) * (x - y)
        picks = []
        umax, k = -1.0, 0
        for j in range(nci):
            if abs(up[j]) > umax:
                umax, k = up[j], j
        picks.append(k)
        for _ in range(2):
            umax, k = -1.0, 0
            for j in range(nci):
                if up[j] > umax and j not in picks:
                    umax, k = up[j], j
            picks.append(k)
        for q, j in enumerate(picks):
            val[r, q] = x[j] ** 2 - y[j] ** 2 if Y is not None else x[j]
            oi[r, q] = res.iconf[j, 0] + 1
            oa[r, q] = res.iconf[j, 1] + res.no + 1
    return val, oi, oa


def stda_uks(xyz4, C, eps, occ, csp, iaoat, S, Lao, Vao, Mao, p: Params, want_A=True):
    """UKS sTDA / sTD-DFT in FP64, restating ``sutda`` (sutda.f:54-1788).

    ``csp`` (nmo) is the spin of each MO (1 alpha, 2 beta).  Per spin: the
    active window (sutda.f:178-360; occupied occ > 0.99 above
    vmin - deps, virtual occ < 0.01 below omax + deps, both limits over all
    MOs), Loewdin MOs, charges, the diagonal A(ia,ia) = de - (ii|aa) + (ia|ia)
    (ak = 1, UCIS) with the K-shift and the SOMO shift (``somo_shift``,
    sutda.f:2402-2422), primaries sorted by energy within their spin.
    ``ptselect_uks`` (sutda.f:1822-2030): every candidate couples to the
    primaries of its own spin by (ia|jb) - (ij|ab) and to those of the other
    spin by (ia|jb) alone; selected alpha / beta candidates are appended to
    their spin's list.  CSF order: alpha block, then beta block.  A
    (``utdamat`` :2311-2399), A+B / A-B (``urpamat`` :2036-2305: cross-spin
    blocks 2(ia|jb) and 0), properties without a spin factor, the velocity
    correction (``utdacorr`` apbtrafo.f:645-750, ``apbtrafo_uks`` :318-574).

    Result: ``iconf`` rows (i, a) index the spin's active occupied / virtual
    MOs (0-based); ``extras['spin']`` (nci) gives 1 / 2 per CSF;
    ``extras['no'], ['nv']`` the per-spin counts ((noa, nob), (nva, nvb)).
    Active MOs of each spin are sorted occupied and virtual separately (as the
    restricted oracle does, stda.f:333 note).
    """
    res = Result()
    res.extras["uks"] = True
    ncent = xyz4.shape[1]
    thr = p.e_thr_ev / EH2EV_IN
    fthr = p.fthr_ev / EH2EV_IN if p.fthr_ev < 1.79e308 else np.inf
    Z = np.rint(xyz4[3]).astype(int)
    res.xmolw = float(np.sum(AMS[Z - 1]))
    csp = np.asarray(csp)
    deps = 2.0 * (1.0 + 0.8 * p.ax) * thr
    occm, virm = occ > 0.99, occ < 0.01
    omax = eps[occm].max() if occm.any() else -1e42
    vmin = eps[virm].min() if virm.any() else 1e42
    othr, vthr = vmin - deps, deps + omax
    nuhf = int(np.sum(occm & (csp == 1))) - int(np.sum(occm & (csp == 2)))
    ak = 1.0
    alpha_k, beta_j = default_alpha_beta(p)
    gj, gk = gamma_matrices(xyz4, p.ax, alpha_k, beta_j)

    spins = []
    for s in (1, 2):
        oidx = np.nonzero(occm & (csp == s) & (eps > othr))[0]
        vidx = np.nonzero(virm & (csp == s) & (eps < vthr))[0]
        oo = oidx[np.argsort(eps[oidx], kind="stable")]
        vv = vidx[np.argsort(eps[vidx], kind="stable")]
        no, nv = len(oo), len(vv)
        Cact = C[:, np.concatenate([oo, vv])]
        epsi = np.concatenate([eps[oo], eps[vv]])
        Co, Cv = Cact[:, :no], Cact[:, no:]
        mu = {name: np.stack([mo_ov(mat[d], Co, Cv) for d in range(3)])
              for name, mat in (("L", Lao), ("V", Vao), ("M", Mao))}
        Clow = lowdin_orthogonal_mos(S, Cact)
        io_all, ia_all = np.meshgrid(np.arange(no), np.arange(nv), indexing="ij")
        io_all, ia_all = io_all.ravel(), ia_all.ravel()
        qii = charges(Clow, iaoat, ncent, np.arange(no), np.arange(no))
        qaa = charges(Clow, iaoat, ncent, no + np.arange(nv), no + np.arange(nv))
        uci = qaa.T @ (gj @ qii)
        qia = charges_block(Clow, iaoat, ncent, np.arange(no), no + np.arange(nv))
        pia = gk @ qia
        ek = np.einsum("Ak,Ak->k", pia, qia)
        de = (epsi[no + ia_all] - epsi[io_all]) - uci[ia_all, io_all] + ak * ek
        if p.kshift:
            sau = p.shftmax * 0.036749320
            wau = p.shftwidth * 0.036749320
            de = de + sau / (1.0 + (ek / wau) ** p.shftsteep)     # kshift_to_ediag
            nsomo = no - nuhf if s == 1 else no + nuhf            # sutda.f:700, 785
            io1, iv1 = io_all + 1, no + ia_all + 1                # 1-based within the spin
            somo = (io1 > nsomo) | (iv1 <= nsomo)
            sau2 = p.shftmax_somo * 0.036749320
            wau2 = p.shftwidth * 0.036749320 * 5.0
            de = np.where(somo, de + sau2 / (1.0 + (ek / wau2) ** p.shftsteep), de)
        pk = np.nonzero(de <= thr)[0]
        ck = np.nonzero((de > thr) & (de < fthr))[0]
        pk = pk[np.argsort(de[pk], kind="stable")]
        qoo = charges_block(Clow, iaoat, ncent, np.arange(no), np.arange(no)).reshape(ncent, no, no)
        qvv = charges_block(Clow, iaoat, ncent, no + np.arange(nv),
                            no + np.arange(nv)).reshape(ncent, nv, nv)
        poo = (gj @ qoo.reshape(ncent, -1)).reshape(qoo.shape)
        spins.append(dict(no=no, nv=nv, oo=oo, vv=vv, epsi=epsi, mu=mu, io=io_all, ia=ia_all,
                          qia=qia, pia=pia, ek=ek, de=de, pk=pk, ck=ck, ed=de[pk].copy(),
                          poo=poo, qvv=qvv))
    A_, B_ = spins
    if (A_["no"] == 0 or A_["nv"] == 0) and (B_["no"] == 0 or B_["nv"] == 0):
        raise OracleError("no CSF, increase energy threshold (-e option)")
    if len(A_["pk"]) + len(B_["pk"]) < 1:
        raise OracleError("No CSF, increase energy threshold (-e option)")

    def coupling(sr, kr, sc, kc):
        """(ia|jb) - delta_{spin} (ij|ab) between CSFs kr of spin sr and kc of sc."""
        R, Cc = spins[sr], spins[sc]
        K = R["pia"][:, kr].T @ Cc["qia"][:, kc]
        if sr != sc:
            return ak * K
        i1, a1, i2, a2 = R["io"][kr], R["ia"][kr], R["io"][kc], R["ia"][kc]
        J = np.einsum("Auv,Auv->uv", R["poo"][:, i1[:, None], i2[None, :]],
                      R["qvv"][:, a1[:, None], a2[None, :]])
        return ak * K - J

    # ptselect_uks: alpha candidates, then beta candidates
    pt2 = [np.zeros(len(A_["pk"])), np.zeros(len(B_["pk"]))]
    new = []
    for s in (0, 1):
        S_ = spins[s]
        ck = S_["ck"]
        incl = np.zeros(len(ck), dtype=bool)
        for q, k in enumerate(ck):
            pts = []
            for t in (0, 1):
                T_ = spins[t]
                if len(T_["pk"]) == 0:
                    pts.append(np.zeros(0))
                    continue
                amat = coupling(s, np.array([k]), t, T_["pk"])[0]
                pts.append(amat ** 2 / (S_["de"][k] - T_["ed"] + 1e-10))
            pert = pts[0].sum() + pts[1].sum()
            if pert > p.thrp:
                incl[q] = True
            else:
                pt2[0] += pts[0]
                pt2[1] += pts[1]
        new.append(ck[incl])
    res.extras["nuhf"] = nuhf
    blocks = []
    for s in (0, 1):
        S_ = spins[s]
        ks = np.concatenate([S_["pk"], new[s]])
        eds = np.concatenate([S_["ed"] - pt2[s], S_["de"][new[s]]])
        blocks.append((ks, eds))
    res.nex = len(A_["pk"]) + len(B_["pk"])
    res.nexpt = len(A_["ck"]) + len(B_["ck"])
    res.new = len(new[0]) + len(new[1])
    (ka, eda), (kb, edb) = blocks
    nexa, nexb = len(ka), len(kb)
    nci = nexa + nexb
    res.iconf = np.concatenate([np.stack([A_["io"][ka], A_["ia"][ka]], axis=1),
                                np.stack([B_["io"][kb], B_["ia"][kb]], axis=1)]).astype(int)
    res.ed = np.concatenate([eda, edb])
    res.pt2 = np.concatenate([pt2[0], pt2[1]])
    spin = np.concatenate([np.ones(nexa, dtype=int), np.full(nexb, 2)])
    res.extras.update(spin=spin, no=(A_["no"], B_["no"]), nv=(A_["nv"], B_["nv"]),
                      nexa=nexa, nexb=nexb)
    res.no, res.nv = A_["no"] + B_["no"], A_["nv"] + B_["nv"]
    if not want_A:
        return res

    # A (utdamat), blocks [alpha, beta]
    sl = [slice(0, nexa), slice(nexa, nci)]
    kk = [ka, kb]
    A = np.zeros((nci, nci))
    Kov = np.zeros((nci, nci))
    Kx = np.zeros((nci, nci))
    for s in (0, 1):
        for t in (0, 1):
            if len(kk[s]) == 0 or len(kk[t]) == 0:
                continue
            A[sl[s], sl[t]] = coupling(s, kk[s], t, kk[t])
            Kov[sl[s], sl[t]] = spins[s]["pia"][:, kk[s]].T @ spins[t]["qia"][:, kk[t]]
        S_ = spins[s]
        if len(kk[s]):
            # (ib|ja) within the spin (exchange type, rrpamat / utdacorr)
            i1, a1 = S_["io"][kk[s]], S_["ia"][kk[s]]
            nv_s = S_["nv"]
            kib = i1[:, None] * nv_s + a1[None, :]
            kja = i1[None, :] * nv_s + a1[:, None]
            Kx[sl[s], sl[s]] = np.einsum("Auv,Auv->uv", S_["pia"][:, kib], S_["qia"][:, kja])
    np.fill_diagonal(A, res.ed)
    Kd = np.concatenate([A_["ek"][ka], B_["ek"][kb]])
    mL = np.concatenate([A_["mu"]["L"][:, A_["io"][ka], A_["ia"][ka]],
                         B_["mu"]["L"][:, B_["io"][kb], B_["ia"][kb]]], axis=1)
    mV = np.concatenate([A_["mu"]["V"][:, A_["io"][ka], A_["ia"][ka]],
                         B_["mu"]["V"][:, B_["io"][kb], B_["ia"][kb]]], axis=1)
    mM = np.concatenate([A_["mu"]["M"][:, A_["io"][ka], A_["ia"][ka]],
                         B_["mu"]["M"][:, B_["io"][kb], B_["ia"][kb]]], axis=1)
    if p.rpa:
        Apb = 2.0 * Kov - p.ax * Kx - (Kov - A)
        Amb = p.ax * Kx - (Kov - A)
        np.fill_diagonal(Apb, res.ed - p.ax * Kd + Kd)
        np.fill_diagonal(Amb, res.ed - Kd + p.ax * Kd)
        if abs(p.ax) < 1e-6:
            Amb = np.diag(res.ed - Kd)
        res.Apb, res.Amb = Apb, Amb
        e, U = np.linalg.eigh(Amb)
        if e[0] < 0:
            raise OracleError("matrix power impossible")
        Ambh = (U * np.sqrt(e)) @ U.T
        w, Zv = sla.eigh(Ambh @ Apb @ Ambh, subset_by_value=(0.0, thr * thr))
        if len(w) < 1:
            raise OracleError("internal error in diag")
        om = np.sqrt(w)
        XpY = (Ambh @ Zv) / np.sqrt(om)
        XmY = (Apb @ XpY) / om
        X = 0.5 * (XpY + XmY)
        res.omega, res.X, res.Y = om, X, XpY - X
        uu, pp = XpY, XmY
    else:
        res.A = A
        w, Xv = sla.eigh(A, subset_by_value=(0.0, thr))
        if len(w) < 1:
            raise OracleError("internal error in diag")
        res.omega, res.X = w, Xv
        uu = pp = Xv
    om = res.omega
    ef = 1.0 / (om + 1e-8)
    tl, tv, tm = mL @ uu, mV @ pp, mM @ pp
    res.fL = om * (2.0 / 3.0) * np.sum(tl * tl, axis=0)
    res.fV = ef * (2.0 / 3.0) * np.sum(tv * tv, axis=0)
    res.RL = ROT_FAC * np.sum(tl * tm, axis=0)
    res.RV = ROT_FAC * np.sum(tv * tm, axis=0) * ef
    res.alpha0 = 2.0 * np.array([np.sum(tl[0] * tl[0] * ef), np.sum(tl[0] * tl[1] * ef),
                                 np.sum(tl[1] * tl[1] * ef), np.sum(tl[0] * tl[2] * ef),
                                 np.sum(tl[1] * tl[2] * ef), np.sum(tl[2] * tl[2] * ef)])
    if (not p.rpa) and p.velcorr:
        Bh = 0.5 * Kov - 0.5 * p.ax * Kx
        np.fill_diagonal(Bh, 0.5 * (Kd - p.ax * Kd))
        Xn = (Bh @ res.X) * ef[None, :]
        xl, xv, xm = mL @ res.X, mV @ res.X, mM @ res.X
        xv2, xm2 = mV @ Xn, mM @ Xn
        hilf = 1.0 - np.exp(-150.0 * om * om)
        efmod = 1.0 / (om ** hilf + 1e-8)
        res.RV = ROT_FAC * np.sum(xv * xm + xv2 * xm + xv * xm2, axis=0) * efmod
    return res

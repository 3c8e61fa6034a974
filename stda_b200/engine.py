"""Host-side binding of the std2g C ABI (``include/std2g.h``).

This is the Python mirror of the reference's call ``stda(...)``
(``stda.f:53-54``, called at ``main.f:928``): the same inputs (MOs, energies,
occupations, AO->atom map, keyword values) and the same outputs (roots, f_L,
f_V, R_L, R_V and ``tda.dat``).  All arithmetic happens in the CUDA library
``libstd2g.so`` built in-tree; when that library is missing this module
raises instead of computing anything on the CPU.
"""
from __future__ import annotations

import ctypes as C
import os
from dataclasses import dataclass, field

import numpy as np

from .integrals import ao_integrals, pack_lower

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libstd2g.so")

STATUS = {
    0: "OK", 1: "EINVAL", 2: "ECUDA", 3: "ENOMEM", 4: "ENOCSF", 5: "ES_NOT_PD",
    6: "EMONORM", 7: "ENOROOT", 8: "ENOCONV", 9: "EAMB_NOT_PD", 10: "ESTATE",
    11: "ECAP", 12: "ENODEV", 13: "ETIMEOUT",
}

EXPORTS = [
    "std2g_create", "std2g_load", "std2g_solve", "std2g_polarizability",
    "std2g_get_csf", "std2g_get_vectors", "std2g_phase_times", "std2g_phase_name",
    "std2g_kernel_launches", "std2g_kernel_stats", "std2g_solver_stats", "std2g_error_string",
    "std2g_destroy", "std2g_screen_noalloc", "std2g_server_create", "std2g_server_submit",
    "std2g_server_poll", "std2g_server_wait", "std2g_server_stats", "std2g_server_destroy",
    "std2g_symeig_check", "std2g_set_sm_limit", "std2g_hyperpolarizability", "std2g_two_photon",
    "std2g_ao_integrals", "std2g_load_prims", "std2g_dgemm_check", "std2g_set_spins",
    "std2g_set_gemm_timing", "std2g_gemm_stats", "std2g_batch_create", "std2g_attach_batch",
    "std2g_batch_stats", "std2g_batch_destroy", "std2g_last_batched", "std2g_server_batch_stats",
]


class Std2gError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"{STATUS.get(code, code)}: {msg}")
        self.code = code
        self.name = STATUS.get(code, str(code))


class Opts(C.Structure):
    _fields_ = [("device", C.c_int), ("precision", C.c_int), ("verbose", C.c_int),
                ("flags", C.c_int), ("max_device_bytes", C.c_int64)]


FLAG_TENSOR_ALWAYS = 1
FLAG_LIBRARY_FP64 = 2   # FP64 products through cuBLAS (library baseline)
FLAG_BATCH_EIGEN = 4    # request server: the slots share one batched eigensolver


class Params(C.Structure):
    _fields_ = [("ax", C.c_double), ("e_thr_ev", C.c_double), ("thrp", C.c_double),
                ("alpha_k", C.c_double), ("beta_j", C.c_double), ("fthr_ev", C.c_double),
                ("triplet", C.c_int), ("rpa", C.c_int), ("velcorr", C.c_int), ("kshift", C.c_int),
                ("shftmax", C.c_double), ("shftwidth", C.c_double), ("shftsteep", C.c_double),
                ("nroots", C.c_int), ("solver", C.c_int), ("conv_tol", C.c_double),
                ("shftmax_somo", C.c_double)]


class ServerOpts(C.Structure):
    _fields_ = [("device", C.c_int), ("precision", C.c_int), ("slots", C.c_int),
                ("trace", C.c_int), ("hbm_budget", C.c_int64), ("flags", C.c_int)]


class Request(C.Structure):
    _fields_ = [("ncent", C.c_int), ("nmo", C.c_int), ("nao", C.c_int),
                ("xyz", C.POINTER(C.c_double)), ("C", C.POINTER(C.c_double)),
                ("eps", C.POINTER(C.c_double)), ("occ", C.POINTER(C.c_double)),
                ("iaoat", C.POINTER(C.c_int)), ("S", C.POINTER(C.c_double)),
                ("mu_L", C.POINTER(C.c_double)), ("mu_V", C.POINTER(C.c_double)),
                ("mu_M", C.POINTER(C.c_double)), ("params", Params), ("nomega", C.c_int),
                ("omega", C.POINTER(C.c_double)), ("nprims", C.c_int),
                ("ipty", C.POINTER(C.c_int)), ("ipao", C.POINTER(C.c_int)),
                ("ipat", C.POINTER(C.c_int)), ("exip", C.POINTER(C.c_double)),
                ("cxip", C.POINTER(C.c_double))]


class Result(C.Structure):
    _fields_ = [("cap", C.c_int), ("nroot", C.c_int), ("no", C.c_int), ("nv", C.c_int),
                ("nex", C.c_int), ("nexpt", C.c_int), ("new_pt", C.c_int), ("nci", C.c_int),
                ("omega", C.POINTER(C.c_double)), ("fL", C.POINTER(C.c_double)),
                ("fV", C.POINTER(C.c_double)), ("RL", C.POINTER(C.c_double)),
                ("RV", C.POINTER(C.c_double)), ("resid", C.POINTER(C.c_double)),
                ("alpha0", C.c_double * 6), ("csf_hash", C.c_uint64), ("ms_total", C.c_double),
                ("dom_coef", C.POINTER(C.c_double)), ("dom_i", C.POINTER(C.c_int)),
                ("dom_a", C.POINTER(C.c_int)), ("err_est", C.POINTER(C.c_double))]


class _ResultBuffers:
    """Host arrays behind one std2g_result (cap roots)."""

    def __init__(self, cap: int):
        self.cap = cap
        self.d = [np.zeros(cap) for _ in range(7)]      # omega fL fV RL RV resid err_est
        self.dc = np.zeros(3 * cap)
        self.di = np.zeros(3 * cap, dtype=np.int32)
        self.da = np.zeros(3 * cap, dtype=np.int32)
        self.res = Result()
        r = self.res
        r.cap = cap
        r.omega, r.fL, r.fV, r.RL, r.RV, r.resid, r.err_est = (_dp(x) for x in self.d)
        r.dom_coef = _dp(self.dc)
        r.dom_i = self.di.ctypes.data_as(C.POINTER(C.c_int))
        r.dom_a = self.da.ctypes.data_as(C.POINTER(C.c_int))

    def solution(self, velo: bool, xmolw: float = 0.0):
        r, n = self.res, self.res.nroot
        return Solution(omega=self.d[0][:n].copy(), fL=self.d[1][:n].copy(),
                        fV=self.d[2][:n].copy(), RL=self.d[3][:n].copy(), RV=self.d[4][:n].copy(),
                        alpha0=np.array(r.alpha0[:]), no=r.no, nv=r.nv, nex=r.nex,
                        nexpt=r.nexpt, new=r.new_pt, nci=r.nci, csf_hash=r.csf_hash,
                        ms=r.ms_total, velo=velo, xmolw=xmolw,
                        extras=dict(resid=self.d[5][:n].copy(), err_est=self.d[6][:n].copy(),
                                    dominant=dict(value=self.dc[:3 * n].reshape(n, 3).copy(),
                                                  i=self.di[:3 * n].reshape(n, 3).copy(),
                                                  a=self.da[:3 * n].reshape(n, 3).copy())))


_lib = None


def library():
    """Load ``libstd2g.so`` (built in-tree); raise if it is absent."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is not built; run stda_b200.build.build()")
        lib = C.CDLL(LIB_PATH)
        dp = C.POINTER(C.c_double)
        ip = C.POINTER(C.c_int)
        lib.std2g_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(Opts)]
        lib.std2g_load.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, dp, dp, dp, dp, ip,
                                   dp, dp, dp, dp]
        lib.std2g_ao_integrals.argtypes = [C.c_void_p, C.c_int, dp, C.c_int, C.c_int, ip, ip, ip,
                                           dp, dp, dp, dp, dp, dp]
        lib.std2g_load_prims.argtypes = [C.c_void_p, C.c_int, C.c_int, C.c_int, dp, dp, dp, dp,
                                         C.c_int, ip, ip, ip, dp, dp]
        lib.std2g_set_spins.argtypes = [C.c_void_p, C.POINTER(C.c_int)]
        lib.std2g_solve.argtypes = [C.c_void_p, C.POINTER(Params), C.POINTER(Result)]
        lib.std2g_polarizability.argtypes = [C.c_void_p, C.POINTER(Params), dp, C.c_int, dp, dp]
        lib.std2g_hyperpolarizability.argtypes = [C.c_void_p, C.POINTER(Params), dp, C.c_int, dp,
                                                  dp]
        lib.std2g_two_photon.argtypes = [C.c_void_p, C.POINTER(Params), C.c_int, dp]
        lib.std2g_get_csf.argtypes = [C.c_void_p, ip, dp, C.c_int, ip]
        lib.std2g_get_vectors.argtypes = [C.c_void_p, dp, dp, C.c_int, ip, ip]
        lib.std2g_phase_times.argtypes = [C.c_void_p, dp, C.c_int]
        lib.std2g_phase_name.argtypes = [C.c_int]
        lib.std2g_phase_name.restype = C.c_char_p
        lib.std2g_kernel_launches.argtypes = [C.c_void_p]
        lib.std2g_kernel_launches.restype = C.c_int64
        lib.std2g_kernel_stats.argtypes = [C.c_void_p, dp, C.POINTER(C.c_int64), dp]
        lib.std2g_set_gemm_timing.argtypes = [C.c_void_p, C.c_int]
        lib.std2g_gemm_stats.argtypes = [C.c_void_p, dp, C.POINTER(C.c_int64), dp]
        lib.std2g_solver_stats.argtypes = [C.c_void_p, ip, C.POINTER(C.c_int64),
                                            C.POINTER(C.c_int64), C.POINTER(C.c_int64)]
        lib.std2g_server_create.argtypes = [C.POINTER(C.c_void_p), C.POINTER(ServerOpts)]
        lib.std2g_server_submit.argtypes = [C.c_void_p, C.POINTER(Request),
                                            C.POINTER(C.c_int64)]
        lib.std2g_server_poll.argtypes = [C.c_void_p, C.c_int64, ip]
        lib.std2g_server_wait.argtypes = [C.c_void_p, C.c_int64, C.POINTER(Result), dp, dp, dp]
        lib.std2g_server_stats.argtypes = [C.c_void_p, C.POINTER(C.c_int64)]
        lib.std2g_set_sm_limit.argtypes = [C.c_void_p, C.c_int]
        lib.std2g_dgemm_check.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                          C.c_double, dp, C.c_int64, dp, C.c_int64, C.c_double,
                                          dp, C.c_int64, C.c_int, dp]
        lib.std2g_symeig_check.argtypes = [C.c_int, C.c_int, C.c_int, dp, dp, dp, dp]
        lib.std2g_server_destroy.argtypes = [C.c_void_p]
        lib.std2g_server_destroy.restype = None
        i64p = C.POINTER(C.c_int64)
        lib.std2g_server_batch_stats.argtypes = [C.c_void_p, i64p, i64p, i64p, dp]
        lib.std2g_batch_create.argtypes = [C.c_int, C.POINTER(C.c_void_p)]
        lib.std2g_attach_batch.argtypes = [C.c_void_p, C.c_void_p]
        lib.std2g_batch_stats.argtypes = [C.c_void_p, i64p, i64p, i64p, dp]
        lib.std2g_batch_destroy.argtypes = [C.c_void_p]
        lib.std2g_batch_destroy.restype = None
        lib.std2g_last_batched.argtypes = [C.c_void_p]
        lib.std2g_screen_noalloc.argtypes = [C.c_int, C.c_int, C.c_int, C.c_int, C.c_int,
                                              C.c_void_p, C.c_void_p, C.c_void_p, C.c_void_p,
                                              C.POINTER(Params), C.c_void_p, C.c_void_p,
                                              C.c_void_p]
        lib.std2g_error_string.argtypes = [C.c_int]
        lib.std2g_error_string.restype = C.c_char_p
        lib.std2g_destroy.argtypes = [C.c_void_p]
        lib.std2g_destroy.restype = None
        _lib = lib
    return _lib


def _dp(a):
    return a.ctypes.data_as(C.POINTER(C.c_double))


def _check(code):
    if code != 0:
        raise Std2gError(code, library().std2g_error_string(code).decode())


@dataclass
class Keywords:
    """std2 keywords of the sTDA path (``main.f:84-131``)."""
    ax: float = 0.5
    e_thr_ev: float = 7.0
    thrp: float = 1e-4
    alpha_k: float = -100.0
    beta_j: float = -100.0
    fthr_ev: float = 1.7976931348623157e308
    triplet: bool = False
    rpa: bool = False
    velcorr: bool = True
    kshift: bool = False
    shftmax: float = 0.5
    shftwidth: float = 0.1
    shftsteep: float = 4.0
    nroots: int = 0
    solver: int = 0
    conv_tol: float = 0.0
    shftmax_somo: float = 1.0

    def to_c(self) -> Params:
        return Params(self.ax, self.e_thr_ev, self.thrp, self.alpha_k, self.beta_j, self.fthr_ev,
                      int(self.triplet), int(self.rpa), int(self.velcorr), int(self.kshift),
                      self.shftmax, self.shftwidth, self.shftsteep, int(self.nroots),
                      int(self.solver), float(self.conv_tol), float(self.shftmax_somo))


@dataclass
class Solution:
    omega: np.ndarray
    fL: np.ndarray
    fV: np.ndarray
    RL: np.ndarray
    RV: np.ndarray
    alpha0: np.ndarray
    no: int
    nv: int
    nex: int
    nexpt: int
    new: int
    nci: int
    csf_hash: int
    ms: float
    velo: bool
    xmolw: float = 0.0
    extras: dict = field(default_factory=dict)


@dataclass
class BoundaryInputs:
    """The arrays that cross the C ABI for one wavefunction."""
    xyz4: np.ndarray     # (ncent, 4) rows x,y,z,Z == Fortran xyz(4,ncent)
    C: np.ndarray        # Fortran-ordered (nao, nmo)
    eps: np.ndarray
    occ: np.ndarray
    iaoat1: np.ndarray   # 1-based int32
    S: np.ndarray        # packed
    muL: np.ndarray      # (3, npk)
    muV: np.ndarray
    muM: np.ndarray

    @property
    def ncent(self):
        return self.xyz4.shape[0]

    @property
    def nao(self):
        return self.C.shape[0]

    @property
    def nmo(self):
        return self.C.shape[1]


def boundary_inputs(mol, ints=None) -> BoundaryInputs:
    """Pack a molecule and its AO integrals into the boundary layout."""
    S, L, V, M = ints if ints is not None else ao_integrals(mol)
    xyz4 = np.ascontiguousarray(np.hstack([mol.xyz, mol.Z[:, None].astype(np.float64)]))
    return BoundaryInputs(
        xyz4=xyz4, C=np.asfortranarray(mol.C), eps=np.ascontiguousarray(mol.eps, dtype=np.float64),
        occ=np.ascontiguousarray(mol.occ, dtype=np.float64),
        iaoat1=np.ascontiguousarray(mol.iaoat() + 1, dtype=np.int32),
        S=pack_lower(S), muL=np.ascontiguousarray(pack_lower(L)),
        muV=np.ascontiguousarray(pack_lower(V)), muM=np.ascontiguousarray(pack_lower(M)))


@dataclass
class Primitives:
    """The primitive list of std2's readers (readbasmold.f:330-517,
    readxtb.f:150-160): per primitive its Cartesian type (1..20), AO and atom
    (1-based), exponent and coefficient with every normalisation folded in."""
    ipty: np.ndarray
    ipao: np.ndarray
    ipat: np.ndarray
    exip: np.ndarray
    cxip: np.ndarray

    @property
    def nprims(self):
        return len(self.ipty)


# Cartesian exponents -> the reference's primitive type (intpack.f90:1213-1218)
_CART_TYPE = {(0, 0, 0): 1, (1, 0, 0): 2, (0, 1, 0): 3, (0, 0, 1): 4, (2, 0, 0): 5,
              (0, 2, 0): 6, (0, 0, 2): 7, (1, 1, 0): 8, (1, 0, 1): 9, (0, 1, 1): 10,
              (3, 0, 0): 11, (0, 3, 0): 12, (0, 0, 3): 13, (2, 1, 0): 14, (2, 0, 1): 15,
              (1, 2, 0): 16, (0, 2, 1): 17, (1, 0, 2): 18, (0, 1, 2): 19, (1, 1, 1): 20}


def primitives(mol) -> Primitives:
    """The primitive list of a molecule's contracted Cartesian basis (AO order
    and normalisation of :meth:`~stda_b200.molden.Molecule.ao_functions`)."""
    ipty, ipao, ipat, exip, cxip = [], [], [], [], []
    for k, (atom, lmn, exps, c) in enumerate(mol.ao_functions()):
        for a, cc in zip(exps, c):
            ipty.append(_CART_TYPE[tuple(lmn)])
            ipao.append(k + 1)
            ipat.append(atom + 1)
            exip.append(float(a))
            cxip.append(float(cc))
    i32 = lambda v: np.ascontiguousarray(v, dtype=np.int32)  # noqa: E731
    f64 = lambda v: np.ascontiguousarray(v, dtype=np.float64)  # noqa: E731
    return Primitives(i32(ipty), i32(ipao), i32(ipat), f64(exip), f64(cxip))


@dataclass
class PrimInputs:
    """A wavefunction with its primitive list instead of AO integrals (the
    served form's std2g_load_prims requests)."""
    xyz4: np.ndarray
    C: np.ndarray
    eps: np.ndarray
    occ: np.ndarray
    prims: Primitives

    @property
    def ncent(self):
        return self.xyz4.shape[0]

    @property
    def nao(self):
        return self.C.shape[0]

    @property
    def nmo(self):
        return self.C.shape[1]


def prim_inputs(mol) -> PrimInputs:
    """Pack a molecule with MOs and its primitive list (no host integrals)."""
    xyz4 = np.ascontiguousarray(np.hstack([mol.xyz, mol.Z[:, None].astype(np.float64)]))
    return PrimInputs(xyz4, np.asfortranarray(mol.C, dtype=np.float64),
                      np.ascontiguousarray(mol.eps, dtype=np.float64),
                      np.ascontiguousarray(mol.occ, dtype=np.float64), primitives(mol))


class Engine:
    """One std2g context on one device (``precision`` 0: FP64, 1: mixed)."""

    def __init__(self, device: int = 0, precision: int = 0, verbose: int = 0, flags: int = 0):
        self.lib = library()
        self.ctx = C.c_void_p()
        opts = Opts(device, precision, verbose, flags, 0)
        _check(self.lib.std2g_create(C.byref(self.ctx), C.byref(opts)))
        self.precision = precision
        self.inputs = None
        self.xmolw = 0.0

    def close(self):
        if self.ctx:
            self.lib.std2g_destroy(self.ctx)
            self.ctx = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def load(self, b: BoundaryInputs):
        self.inputs = b
        from .tdadat import molecular_mass
        self.xmolw = molecular_mass(b.xyz4[:, 3])
        _check(self.lib.std2g_load(
            self.ctx, b.ncent, b.nmo, b.nao, _dp(b.xyz4), _dp(b.C), _dp(b.eps), _dp(b.occ),
            b.iaoat1.ctypes.data_as(C.POINTER(C.c_int)), _dp(b.S), _dp(b.muL), _dp(b.muV),
            _dp(b.muM)))

    def ao_integrals(self, xyz4, nao: int, pr: Primitives):
        """Packed S, mu_L, mu_V, mu_M (std2g_load layout) formed on the device."""
        npk = nao * (nao + 1) // 2
        S, L, V, M = np.zeros(npk), np.zeros(3 * npk), np.zeros(3 * npk), np.zeros(3 * npk)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
        xyz4 = np.ascontiguousarray(xyz4, dtype=np.float64)
        _check(self.lib.std2g_ao_integrals(self.ctx, xyz4.shape[0], _dp(xyz4), nao, pr.nprims,
                                           ip(pr.ipty), ip(pr.ipao), ip(pr.ipat), _dp(pr.exip),
                                           _dp(pr.cxip), _dp(S), _dp(L), _dp(V), _dp(M)))
        return S, L.reshape(3, npk), V.reshape(3, npk), M.reshape(3, npk)

    def load_prims(self, xyz4, C_mo, eps, occ, pr: Primitives):
        """std2g_load_prims: MOs plus the primitive list; integrals on the device."""
        xyz4 = np.ascontiguousarray(xyz4, dtype=np.float64)
        Cf = np.asfortranarray(C_mo, dtype=np.float64)
        eps = np.ascontiguousarray(eps, dtype=np.float64)
        occ = np.ascontiguousarray(occ, dtype=np.float64)
        from .tdadat import molecular_mass
        self.xmolw = molecular_mass(xyz4[:, 3])
        self.inputs = None
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
        _check(self.lib.std2g_load_prims(self.ctx, xyz4.shape[0], Cf.shape[1], Cf.shape[0],
                                         _dp(xyz4), _dp(Cf), _dp(eps), _dp(occ), pr.nprims,
                                         ip(pr.ipty), ip(pr.ipao), ip(pr.ipat), _dp(pr.exip),
                                         _dp(pr.cxip)))

    def set_spins(self, csp):
        """Mark the loaded wavefunction unrestricted: csp[k] = 1 (alpha) or 2
        (beta) per MO (std2g_set_spins)."""
        csp = np.ascontiguousarray(csp, dtype=np.int32)
        _check(self.lib.std2g_set_spins(self.ctx, csp.ctypes.data_as(C.POINTER(C.c_int))))

    def solve(self, kw: Keywords, cap: int = 4096) -> Solution:
        """One solve; ``cap`` is the initial room for roots.  When the window
        holds more roots (``nroots = 0`` on a large CSF space) the library
        reports STD2G_ECAP with the count, and the solve is repeated once with
        that much room."""
        while True:
            rb = _ResultBuffers(cap)
            code = self.lib.std2g_solve(self.ctx, C.byref(kw.to_c()), C.byref(rb.res))
            if code == 11 and rb.res.nroot > cap:
                cap = rb.res.nroot
                continue
            _check(code)
            break
        return rb.solution((not kw.rpa) and kw.velcorr, self.xmolw)

    def polarizability(self, kw: Keywords, omegas):
        om = np.ascontiguousarray(omegas, dtype=np.float64)
        out = np.zeros(len(om) * 9)
        resid = np.zeros(len(om))
        _check(self.lib.std2g_polarizability(self.ctx, C.byref(kw.to_c()), _dp(om), len(om),
                                             _dp(out), _dp(resid)))
        return out.reshape(len(om), 3, 3), resid

    def hyperpolarizability(self, kw: Keywords, wavelengths_nm):
        """beta(-2w; w, w) as lresp1 prints it (linear_response.f:196-700): at
        w = 0 and at w = 45.56335 / lambda for each wavelength (nm).  Returns
        (w in eV as printed, beta [nw, 3, 3, 3], beta_HRS [nw])."""
        om = np.ascontiguousarray([0.0] + [45.56335 / float(w) for w in wavelengths_nm])
        beta = np.zeros((len(om), 3, 3, 3))
        hrs = np.zeros(len(om))
        _check(self.lib.std2g_hyperpolarizability(self.ctx, C.byref(kw.to_c()), _dp(om), len(om),
                                                  _dp(beta), _dp(hrs)))
        return om * 27.21139, beta, hrs

    def two_photon(self, kw: Keywords, ntrans: int):
        """Two-photon absorption of the lowest ``ntrans`` sTD-DFT states as
        lresp_2PA_SP writes its 2PA-abs rows (linear_response.f:4604-4938):
        (n, w_n eV, delta_par, delta_perp, delta_circ, rho) per state."""
        rows = np.zeros((ntrans, 6))
        _check(self.lib.std2g_two_photon(self.ctx, C.byref(kw.to_c()), int(ntrans), _dp(rows)))
        return rows

    def csf(self):
        n = C.c_int()
        _check_cap = self.lib.std2g_get_csf(self.ctx, None, None, 0, C.byref(n))
        if _check_cap not in (0, 11):
            _check(_check_cap)
        iconf = np.zeros(2 * n.value, dtype=np.int32)
        ed = np.zeros(n.value)
        _check(self.lib.std2g_get_csf(self.ctx, iconf.ctypes.data_as(C.POINTER(C.c_int)),
                                      _dp(ed), n.value, C.byref(n)))
        return iconf.reshape(-1, 2), ed

    def vectors(self, rpa=False):
        nr, nci = C.c_int(), C.c_int()
        code = self.lib.std2g_get_vectors(self.ctx, None, None, 0, C.byref(nr), C.byref(nci))
        if code not in (0, 11):
            _check(code)
        X = np.zeros((nr.value, nci.value))
        Y = np.zeros((nr.value, nci.value)) if rpa else None
        _check(self.lib.std2g_get_vectors(self.ctx, _dp(X), _dp(Y) if rpa else None, nr.value,
                                          C.byref(nr), C.byref(nci)))
        return (X.T, Y.T) if rpa else X.T

    def phase_times(self):
        ms = np.zeros(16)
        n = self.lib.std2g_phase_times(self.ctx, _dp(ms), 16)
        return {self.lib.std2g_phase_name(q).decode(): ms[q] for q in range(n)}

    def kernel_stats(self):
        """Tensor-core contraction time / launches / algorithmic FLOPs of the last solve."""
        ms, fl = C.c_double(), C.c_double()
        n = C.c_int64()
        _check(self.lib.std2g_kernel_stats(self.ctx, C.byref(ms), C.byref(n), C.byref(fl)))
        return {"tc_ms": ms.value, "tc_launches": n.value, "tc_flop": fl.value}

    def set_gemm_timing(self, on: bool) -> None:
        """Bracket every FP64 product of later solves with an event pair."""
        _check(self.lib.std2g_set_gemm_timing(self.ctx, int(bool(on))))

    def gemm_stats(self):
        """FP64 products of the last solve: device time (timing on), count, FLOPs."""
        ms, fl = C.c_double(), C.c_double()
        n = C.c_int64()
        _check(self.lib.std2g_gemm_stats(self.ctx, C.byref(ms), C.byref(n), C.byref(fl)))
        return {"ms": ms.value, "calls": n.value, "flop": fl.value}

    def solver_stats(self):
        it = C.c_int()
        mv, mv64, rc = C.c_int64(), C.c_int64(), C.c_int64()
        _check(self.lib.std2g_solver_stats(self.ctx, C.byref(it), C.byref(mv), C.byref(mv64),
                                           C.byref(rc)))
        return {"davidson_iters": it.value, "sigma_vectors_mixed": mv.value,
                "sigma_vectors_fp64": mv64.value, "pt_rechecked_fp64": rc.value}

    def kernel_launches(self):
        return int(self.lib.std2g_kernel_launches(self.ctx))


def stda(mol, kw: Keywords, ints=None, device=0, precision=0):
    """One-call mirror of ``call stda(...)``: returns (Solution, tda.dat text)."""
    from .tdadat import tda_dat
    eng = Engine(device, precision)
    try:
        eng.load(boundary_inputs(mol, ints))
        sol = eng.solve(kw)
    finally:
        eng.close()
    return sol, tda_dat(sol, kw)


class Server:
    """Served form: a request loop with continuous batching over ``slots``
    engine contexts on one device (``include/std2g.h``, served / batched form).

    ``submit`` copies the inputs and returns a ticket at once; ``wait`` blocks
    until that request has finished and returns its roots and properties,
    alpha(omega) when requested, and its queued / running / total times (ms).
    ``trace=True`` prints one line per finished request on stderr (slot,
    requests in flight at its start, SM share, times, phase times).
    """

    def __init__(self, device: int = 0, precision: int = 1, slots: int = 4,
                 hbm_budget: int = 0, trace: bool = False, flags: int = 0):
        self.lib = library()
        self.srv = C.c_void_p()
        _check(self.lib.std2g_server_create(C.byref(self.srv),
                                            C.byref(ServerOpts(device, precision, slots,
                                                               int(bool(trace)),
                                                               int(hbm_budget), int(flags)))))
        self._nomega = {}

    def submit(self, b, kw: Keywords, omegas=None) -> int:
        """Queue one request: ``b`` is a :class:`BoundaryInputs` (packed AO
        integrals from the host) or a :class:`PrimInputs` (primitive list; the
        integrals are formed on the device)."""
        om = None if omegas is None else np.ascontiguousarray(omegas, dtype=np.float64)
        ip = lambda a: a.ctypes.data_as(C.POINTER(C.c_int))  # noqa: E731
        nom = 0 if om is None else len(om)
        omp = None if om is None else _dp(om)
        if isinstance(b, PrimInputs):
            pr = b.prims
            rq = Request(b.ncent, b.nmo, b.nao, _dp(b.xyz4), _dp(b.C), _dp(b.eps), _dp(b.occ),
                         None, None, None, None, None, kw.to_c(), nom, omp, pr.nprims,
                         ip(pr.ipty), ip(pr.ipao), ip(pr.ipat), _dp(pr.exip), _dp(pr.cxip))
        else:
            rq = Request(b.ncent, b.nmo, b.nao, _dp(b.xyz4), _dp(b.C), _dp(b.eps), _dp(b.occ),
                         ip(b.iaoat1), _dp(b.S), _dp(b.muL), _dp(b.muV), _dp(b.muM), kw.to_c(),
                         nom, omp, 0, None, None, None, None, None)
        t = C.c_int64()
        _check(self.lib.std2g_server_submit(self.srv, C.byref(rq), C.byref(t)))
        self._nomega[t.value] = (0 if om is None else len(om), kw)
        return t.value

    def done(self, ticket: int) -> bool:
        d = C.c_int()
        _check(self.lib.std2g_server_poll(self.srv, ticket, C.byref(d)))
        return bool(d.value)

    def wait(self, ticket: int, cap: int = 4096):
        """Block until the request has finished.  A result with more roots
        than ``cap`` keeps its ticket (STD2G_ECAP with the count), and the wait
        is repeated with that much room."""
        nom, kw = self._nomega.pop(ticket)
        alpha = np.zeros(max(1, nom) * 9)
        ares = np.zeros(max(1, nom))
        timing = np.zeros(3)
        while True:
            rb = _ResultBuffers(cap)
            code = self.lib.std2g_server_wait(self.srv, ticket, C.byref(rb.res), _dp(alpha),
                                              _dp(ares), _dp(timing))
            if code == 11 and rb.res.nroot > cap:
                cap = rb.res.nroot
                continue
            _check(code)
            break
        sol = rb.solution((not kw.rpa) and kw.velcorr)
        a = alpha[:nom * 9].reshape(nom, 3, 3) if nom else None
        return sol, a, (ares[:nom] if nom else None), dict(
            queued_ms=timing[0], run_ms=timing[1], latency_ms=timing[2])

    def batch_stats(self) -> dict:
        """The shared batched eigensolver's counters (server flag
        STD2G_FLAG_BATCH_EIGEN): problems solved, batched iterations, and the
        mean number of problems per iteration."""
        pr, it, mem = C.c_int64(), C.c_int64(), C.c_int64()
        ms = np.zeros(2)
        _check(self.lib.std2g_server_batch_stats(self.srv, C.byref(pr), C.byref(it),
                                                 C.byref(mem), _dp(ms)))
        n = max(1, it.value)
        return {"problems": pr.value, "iterations": it.value,
                "mean_batch": mem.value / n, "iteration_ms": ms[0] / n,
                "to_first_sync_ms": ms[1] / n}

    def stats(self) -> dict:
        st = (C.c_int64 * 7)()
        _check(self.lib.std2g_server_stats(self.srv, st))
        keys = ("submitted", "completed", "in_flight", "peak_in_flight", "bytes_in_flight",
                "peak_bytes", "budget")
        return dict(zip(keys, [int(x) for x in st]))

    def close(self):
        if self.srv:
            self.lib.std2g_server_destroy(self.srv)
            self.srv = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def dgemm_check(A, B, Cm, ta=False, tb=False, alpha=1.0, beta=0.0, device: int = 0):
    """The engine's FP64 product on host arrays: A, B, Cm are (batch, rows,
    cols) or 2-D; returns (alpha op(A) op(B) + beta Cm, device ms)."""
    A3, B3, C3 = (np.asfortranarray(x if x.ndim == 3 else x[None]).astype(np.float64)
                  for x in (A, B, Cm))
    batch = A3.shape[0]
    # column-major members laid out one after another
    a = np.concatenate([np.asfortranarray(x).ravel(order="F") for x in A3])
    b = np.concatenate([np.asfortranarray(x).ravel(order="F") for x in B3])
    c = np.concatenate([np.asfortranarray(x).ravel(order="F") for x in C3])
    m, n = C3.shape[1], C3.shape[2]
    k = A3.shape[1] if ta else A3.shape[2]
    ms = np.zeros(1)
    lib = library()
    a = a if a.size else np.zeros(1)
    b = b if b.size else np.zeros(1)
    _check(lib.std2g_dgemm_check(device, int(ta), int(tb), m, n, k, alpha, _dp(a),
                                 max(1, A3.shape[1]), _dp(b), max(1, B3.shape[1]), beta, _dp(c), m,
                                 batch, _dp(ms)))
    out = c.reshape(batch, n, m).transpose(0, 2, 1)
    return (out if Cm.ndim == 3 else out[0]), float(ms[0])


def symeig_check(A, k, device: int = 0):
    """The engine's small symmetric eigensolver (lowest k pairs) and cuSOLVER's
    eigenvalues for the same matrix: (w, Z, w_ref)."""
    A = np.asfortranarray(A, dtype=np.float64)
    n = A.shape[0]
    w, Z, wr = np.zeros(k), np.zeros((n, k), order="F"), np.zeros(n)
    _check(library().std2g_symeig_check(device, n, k, _dp(A), _dp(w), _dp(Z), _dp(wr)))
    return w, Z, wr

"""std2g_screen_noalloc: the diagonal screen for callers that cannot allocate.

Some hosts cannot let this library call cudaMalloc: their GPU memory is
owned by another allocator (a framework that reserved it for its own pool),
or they are at a point where the device synchronisation that cudaMalloc
implies is not allowed.  std2g_screen_noalloc takes device buffers the caller
already owns and keeps its work arrays in a fixed __device__ array.

Checked here, through the C ABI:
* against the allocating entry point std2g_solve: with the PT selection
  switched off (PT limit = E_thr) the diagonal energies std2g_get_csf reports
  are exactly the screen's values for the primary CSFs;
* against the FP64 oracle's diagonal of every (i, a) pair and its primary /
  PT-candidate classification (stda.f:593-640), with a PT limit above E_thr
  so that candidates (flag 2) occur, and with the K-shift of the xTB path;
* two calls in a row agree, and the largest case runs first, so scratch left
  over from a bigger problem cannot leak into the later, smaller ones.
This file is collected last on purpose.
"""
import ctypes as C

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

# largest first: later cases run over the scratch the earlier ones left
CASES = ["cluster_kshift", "benzene_pt", "water"]


def _inputs(mol, ints, kw):
    """Active window, Loewdin MOs and energies as the engine builds them."""
    from oracle.stda_fp64 import EH2EV_IN, lowdin_orthogonal_mos, select_window
    S = ints[0]
    o, v = select_window(mol.eps, mol.occ, kw["ax"], kw["e_thr_ev"] / EH2EV_IN)
    o = o[np.argsort(mol.eps[o], kind="stable")]
    v = v[np.argsort(mol.eps[v], kind="stable")]
    act = np.concatenate([o, v])
    clow = lowdin_orthogonal_mos(S, mol.C[:, act])
    return len(o), len(v), clow, mol.eps[act]


def _case(name, water):
    from stda_b200 import synth
    if name == "water":
        mol, ints = water
        return mol, ints, dict(ax=1.0, e_thr_ev=20.0), None
    if name == "benzene_pt":
        mol, ints = synth.benzene(with_ints=True)
        return mol, ints, dict(ax=0.5, e_thr_ev=10.0), 14.0
    mol, ints = synth.random_molecule(30, seed=3, with_ints=True)
    return mol, ints, dict(ax=0.5, e_thr_ev=8.0, kshift=True), 12.0


@pytest.mark.parametrize("name", CASES)
def test_screen_noalloc_matches_solve_and_oracle(name, water):
    import torch
    from oracle.stda_fp64 import EH2EV_IN, Params, stda as oracle_stda
    from stda_b200.engine import Engine, Keywords, boundary_inputs, library
    mol, ints, kw, fthr = _case(name, water)
    kw_screen = dict(kw, fthr_ev=fthr) if fthr else dict(kw)
    # the allocating path, PT selection off: ed of the primaries = screen values
    eng = Engine(0, 0)
    b = boundary_inputs(mol, ints)
    eng.load(b)
    eng.solve(Keywords(**dict(kw, fthr_ev=kw["e_thr_ev"])))
    iconf, ed = eng.csf()
    eng.close()
    # the FP64 oracle's diagonal of every pair and its classification
    ref = oracle_stda(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), *ints,
                      Params(**kw_screen), want_A=False)
    de_ref = ref.extras["de_all"]
    thr = kw["e_thr_ev"] / EH2EV_IN
    lim = fthr / EH2EV_IN if fthr else np.inf
    flag_ref = np.where(de_ref <= thr, 1, np.where(de_ref < lim, 2, 0))

    no, nv, clow, eps_act = _inputs(mol, ints, kw)
    assert (no, nv) == (ref.no, ref.nv)
    dev = torch.device("cuda:0")
    d_xyz = torch.tensor(b.xyz4, dtype=torch.float64, device=dev)
    d_iaoat = torch.tensor(b.iaoat1, dtype=torch.int32, device=dev)
    d_clow = torch.tensor(np.ascontiguousarray(clow.T), dtype=torch.float64, device=dev)
    d_eps = torch.tensor(eps_act, dtype=torch.float64, device=dev)
    lib = library()
    par = Keywords(**kw_screen).to_c()
    runs = []
    for _ in range(2):
        d_de = torch.full((no * nv,), np.nan, dtype=torch.float64, device=dev)
        d_flag = torch.full((no * nv,), -1, dtype=torch.int32, device=dev)
        code = lib.std2g_screen_noalloc(0, b.ncent, b.nao, no, nv, d_xyz.data_ptr(),
                                        d_iaoat.data_ptr(), d_clow.data_ptr(), d_eps.data_ptr(),
                                        C.byref(par), d_de.data_ptr(), d_flag.data_ptr(), None)
        assert code == 0, lib.std2g_error_string(code)
        torch.cuda.synchronize()
        runs.append((d_de.cpu().numpy(), d_flag.cpu().numpy()))
    (de1, fl1), (de2, fl2) = runs
    assert np.array_equal(de1, de2) and np.array_equal(fl1, fl2)
    # against the oracle: every pair's diagonal and classification
    assert np.abs(de1 - de_ref).max() < 1e-10
    assert np.array_equal(fl1, flag_ref)
    if fthr:
        assert (fl1 == 2).any()
    # against the allocating entry point: the primaries and their energies
    k_solve = (iconf[:, 0] - 1) * nv + (iconf[:, 1] - 1 - no)
    assert np.array_equal(np.sort(k_solve), np.nonzero(fl1 == 1)[0])
    assert np.abs(de1[k_solve] - ed).max() < 1e-10


def test_screen_noalloc_rejects_oversize_and_nulls():
    import torch
    from stda_b200.engine import Keywords, library
    lib = library()
    par = Keywords(ax=0.5, e_thr_ev=7.0).to_c()
    buf = torch.zeros(16, dtype=torch.float64, device="cuda:0")
    p = buf.data_ptr()
    # 3000 atoms x 100 x 100 pairs needs far more than the fixed scratch
    assert lib.std2g_screen_noalloc(0, 3000, 4000, 100, 100, p, p, p, p, C.byref(par), p, p,
                                    None) == 11
    assert lib.std2g_screen_noalloc(0, 3, 7, 5, 2, None, p, p, p, C.byref(par), p, p, None) == 1

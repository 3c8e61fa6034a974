"""CUDA engine vs the FP64 oracle and the reference goldens, through the C ABI.

Tolerances: the FP64 form must agree with the oracle to 1e-8 Eh in every
root and 1e-6 relative in f_L/f_V (different summation orders only); the CSF
selection must be identical (same (i,a) list in the same order).
"""
import json
import os

import numpy as np
import pytest

from oracle.stda_fp64 import Params as OParams
from oracle.stda_fp64 import dynamic_polarizability, stda as oracle_stda
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

EXPECTED = json.load(open(os.path.join(GOLDEN, "reference_expected.json")))


def _engine(precision=0):
    """Mixed-form engines use the tensor-core paths at every size here, so that
    the small test molecules exercise them."""
    from stda_b200.engine import Engine, FLAG_TENSOR_ALWAYS
    return Engine(0, precision, flags=FLAG_TENSOR_ALWAYS if precision == 1 else 0)


def _oracle(mol, ints, **kw):
    S, L, V, M = ints
    return oracle_stda(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), S, L, V, M, OParams(**kw))


def _run(mol, ints, precision=0, **kw):
    from stda_b200.engine import Keywords, boundary_inputs
    eng = _engine(precision)
    eng.load(boundary_inputs(mol, ints))
    sol = eng.solve(Keywords(**kw))
    iconf, ed = eng.csf()
    return eng, sol, iconf, ed


def _same_csf(ref, iconf):
    got = np.stack([iconf[:, 0] - 1, iconf[:, 1] - 1 - ref.no], axis=1)
    return got.shape == ref.iconf.shape and np.array_equal(got, ref.iconf)


@pytest.mark.parametrize("name", ["EXCI_TEST1", "EXCI_TEST2", "EXCI_TEST3"])
def test_water_tda_golden(water, name):
    from stda_b200.engine import Keywords
    from stda_b200.tdadat import tda_dat
    from oracle.stda_fp64 import read_tda_dat
    mol, ints = water
    case = EXPECTED[name]
    eng, sol, iconf, ed = _run(mol, ints, **case["args"])
    got = read_tda_dat(tda_dat(sol, Keywords(**case["args"])))
    exp = np.array(case["rows"])
    assert got.shape == exp.shape
    assert np.abs(got[:, 1:4] - exp[:, 1:4]).max() <= 1e-3
    ref = _oracle(mol, ints, **case["args"])
    assert _same_csf(ref, iconf)
    assert np.abs(sol.omega - ref.omega).max() < 1e-8
    assert np.allclose(sol.fL, ref.fL, rtol=1e-6, atol=1e-10)
    assert np.allclose(sol.RV, ref.RV, rtol=1e-6, atol=1e-8)


@pytest.mark.parametrize("name", ["2PA_TEST1", "2PA_TEST2", "2PA_TEST3"])
def test_water_std_dft_golden(water, name):
    mol, ints = water
    case = EXPECTED[name]
    eng, sol, iconf, ed = _run(mol, ints, rpa=True, **case["args"])
    exp = np.array(case["rows"])
    assert np.abs(sol.omega[:len(exp)] * 27.21139 - exp[:, 1]).max() <= 1e-3
    ref = _oracle(mol, ints, rpa=True, **case["args"])
    assert np.abs(sol.omega - ref.omega).max() < 1e-8
    assert np.allclose(sol.fL, ref.fL, rtol=1e-6, atol=1e-10)


@pytest.fixture(scope="module")
def benzene():
    from stda_b200 import synth
    return synth.benzene(with_ints=True)


def test_benzene_fp64_vs_oracle(benzene):
    mol, ints = benzene
    kw = dict(ax=0.5, e_thr_ev=10.0)
    eng, sol, iconf, ed = _run(mol, ints, **kw)
    ref = _oracle(mol, ints, **kw)
    assert (sol.nex, sol.nexpt, sol.new, sol.nci) == (ref.nex, ref.nexpt, ref.new, len(ref.iconf))
    assert _same_csf(ref, iconf)
    assert np.abs(ed - ref.ed).max() < 1e-10
    assert len(sol.omega) == len(ref.omega)
    assert np.abs(sol.omega - ref.omega).max() < 1e-8
    for a, b in ((sol.fL, ref.fL), (sol.fV, ref.fV), (sol.RL, ref.RL), (sol.RV, ref.RV)):
        assert np.allclose(a, b, rtol=1e-6, atol=1e-9)


def test_benzene_rpa_and_polarizability(benzene):
    from stda_b200.engine import Keywords
    mol, ints = benzene
    kw = dict(ax=0.5, e_thr_ev=10.0)
    eng, sol, iconf, ed = _run(mol, ints, rpa=True, **kw)
    ref = _oracle(mol, ints, rpa=True, **kw)
    assert np.abs(sol.omega - ref.omega).max() < 1e-8
    om = [0.0, 0.03, 0.06, 0.09]
    alpha, resid = eng.polarizability(Keywords(**kw), om)
    aref = dynamic_polarizability(ref, om)
    assert np.allclose(alpha, aref, rtol=1e-8, atol=1e-8)
    assert resid.max() < 1e-10


def test_polarizability_mixed_refinement(benzene):
    """Mixed form of alpha(w): FP32 conjugate gradients inside FP64 iterative
    refinement.  Below the first excitation the FP64 residual must reach 1e-8
    and alpha must match the oracle to 1e-4 relative (it does to ~1e-9); a
    frequency above the first excitation goes through the FP64 form and must
    match it as well."""
    from stda_b200.engine import Keywords
    mol, ints = benzene
    kw = dict(ax=0.5, e_thr_ev=10.0)
    ref = _oracle(mol, ints, rpa=True, **kw)
    eng = _engine(1)
    from stda_b200.engine import boundary_inputs
    eng.load(boundary_inputs(mol, ints))
    above = float(ref.omega[0]) * 1.05           # just above the lowest root
    om = [0.0, 0.03, 0.06, 0.09, above]
    alpha, resid = eng.polarizability(Keywords(**kw), om)
    aref = dynamic_polarizability(ref, om)
    scale = np.abs(aref).max(axis=(1, 2))
    rel = np.abs(alpha - aref).max(axis=(1, 2)) / scale
    assert rel.max() < 1e-4, rel
    assert resid.max() < 1e-8, resid
    # the mixed and FP64 forms agree on a larger molecule
    from stda_b200 import synth
    mol2, ints2 = synth.random_molecule(40, seed=11, with_ints=True)
    kw2 = Keywords(ax=0.5, e_thr_ev=9.0)
    out = []
    for prec in (0, 1):
        e = _engine(prec)
        e.load(boundary_inputs(mol2, ints2))
        out.append(e.polarizability(kw2, [0.0, 0.05, 0.1]))
    (a0, r0), (a1, r1) = out
    rel2 = np.abs(a1 - a0).max(axis=(1, 2)) / np.abs(a0).max(axis=(1, 2))
    assert rel2.max() < 1e-4, rel2
    assert r1.max() < 1e-8
    # matrix-free operators (no n x n storage), both forms, against the dense FP64 form
    kw3 = Keywords(ax=0.5, e_thr_ev=9.0, solver=2)
    for prec in (0, 1):
        e = _engine(prec)
        e.load(boundary_inputs(mol2, ints2))
        a3, r3 = e.polarizability(kw3, [0.0, 0.05, 0.1])
        rel3 = np.abs(a3 - a0).max(axis=(1, 2)) / np.abs(a0).max(axis=(1, 2))
        assert rel3.max() < 1e-6, (prec, rel3)
        assert r3.max() < 1e-8


def test_random_cluster_triplet_and_kshift():
    from stda_b200 import synth
    mol, ints = synth.random_molecule(24, seed=5, with_ints=True)
    for kw in (dict(ax=0.25, e_thr_ev=9.0, triplet=True), dict(ax=0.5, e_thr_ev=8.0, kshift=True),
               dict(ax=0.0, e_thr_ev=8.0, velcorr=False)):
        eng, sol, iconf, ed = _run(mol, ints, **kw)
        ref = _oracle(mol, ints, **kw)
        assert _same_csf(ref, iconf)
        assert np.abs(sol.omega - ref.omega).max() < 1e-8
        assert np.allclose(sol.fL, ref.fL, rtol=1e-6, atol=1e-9)


def test_error_paths(water):
    from stda_b200.engine import Engine, Keywords, Std2gError, boundary_inputs
    mol, ints = water
    eng = Engine(0, 0)
    with pytest.raises(Std2gError) as e:
        eng.solve(Keywords(ax=0.5, e_thr_ev=10.0))
    assert e.value.name == "ESTATE"
    eng.load(boundary_inputs(mol, ints))
    with pytest.raises(Std2gError) as e:
        eng.solve(Keywords(ax=0.5, e_thr_ev=0.01))        # nothing below 0.01 eV
    assert e.value.name in ("ENOCSF", "ENOROOT")
    with pytest.raises(Std2gError) as e:
        eng.solve(Keywords(ax=0.5, e_thr_ev=-1.0))
    assert e.value.name == "EINVAL"
    # the context stays usable after errors
    sol = eng.solve(Keywords(ax=1.0, e_thr_ev=20.0))
    assert len(sol.omega) == 4


@pytest.mark.parametrize("precision", [0, 1])
def test_matrix_free_davidson_vs_oracle(benzene, precision):
    """Lowest roots by the matrix-free blocked Davidson vs the oracle's dense
    diagonalisation, including the velocity-corrected rotatory strengths."""
    mol, ints = benzene
    kw = dict(ax=0.5, e_thr_ev=10.0)
    eng, sol, iconf, ed = _run(mol, ints, precision=precision, nroots=12, solver=2,
                               conv_tol=1e-8, **kw)
    ref = _oracle(mol, ints, **kw)
    assert _same_csf(ref, iconf)
    if precision == 0:
        assert np.abs(sol.omega - ref.omega[:12]).max() < 1e-9
        assert np.allclose(sol.fL, ref.fL[:12], rtol=1e-5, atol=1e-8)
        assert np.allclose(sol.fV, ref.fV[:12], rtol=1e-5, atol=1e-8)
        assert np.allclose(sol.RV, ref.RV[:12], rtol=1e-4, atol=1e-6)
    else:   # split-BF16 tensor-core products (first stage, velocity correction)
        assert np.abs(sol.omega - ref.omega[:12]).max() * 27.21139 < 1e-4
        big = ref.fL[:12] > 1e-3
        assert np.all(np.abs(sol.fL[big] - ref.fL[:12][big]) / ref.fL[:12][big] < 1e-4)
        bigv = ref.fV[:12] > 1e-3   # f_V: velocity correction from the exchange products
        assert np.all(np.abs(sol.fV[bigv] - ref.fV[:12][bigv]) / ref.fV[:12][bigv] < 1e-4)
        assert np.allclose(sol.RV, ref.RV[:12], rtol=1e-3, atol=1e-6)


def test_matrix_free_larger_cluster():
    from stda_b200 import synth
    mol, ints = synth.random_molecule(36, seed=11, with_ints=True)
    kw = dict(ax=0.5, e_thr_ev=8.0)
    eng, sol, iconf, ed = _run(mol, ints, nroots=20, solver=2, conv_tol=1e-8, **kw)
    ref = _oracle(mol, ints, **kw)
    assert _same_csf(ref, iconf)
    n = min(20, len(ref.omega))
    assert n >= 10
    assert np.abs(sol.omega[:n] - ref.omega[:n]).max() < 1e-9
    assert np.allclose(sol.fL[:n], ref.fL[:n], rtol=1e-5, atol=1e-8)
    assert np.allclose(sol.RV[:n], ref.RV[:n], rtol=1e-4, atol=1e-6)


def test_mixed_form_pt_selection_matches_fp64(benzene):
    """Tensor-core (split-BF16) PT selection: same CSF set as the FP64 oracle,
    roots within 1e-4 eV and oscillator strengths within 1e-4 relative."""
    mol, ints = benzene
    kw = dict(ax=0.5, e_thr_ev=10.0)
    eng, sol, iconf, ed = _run(mol, ints, precision=1, **kw)
    ref = _oracle(mol, ints, **kw)
    assert _same_csf(ref, iconf)
    assert np.abs(sol.omega - ref.omega).max() * 27.21139 < 1e-4
    big = ref.fL > 1e-3
    assert np.all(np.abs(sol.fL[big] - ref.fL[big]) / ref.fL[big] < 1e-4)
    assert eng.kernel_stats()["tc_launches"] > 0


@pytest.mark.parametrize("natoms,seed", [(30, 3), (40, 4)])
def test_mixed_form_clusters(natoms, seed):
    from stda_b200 import synth
    mol, ints = synth.random_molecule(natoms, seed=seed, with_ints=True)
    kw = dict(ax=0.5, e_thr_ev=8.0)
    eng, sol, iconf, ed = _run(mol, ints, precision=1, nroots=10, solver=2, conv_tol=1e-7, **kw)
    ref = _oracle(mol, ints, **kw)
    assert _same_csf(ref, iconf)
    n = min(10, len(ref.omega))
    assert np.abs(sol.omega[:n] - ref.omega[:n]).max() * 27.21139 < 1e-4


def test_mixed_small_alpha_runs_the_fp64_solve(benzene):
    """Below the tensor-core gate of the matrix-free alpha(w) solve (atoms x
    CSFs < 1.5e6) the mixed form runs the FP64 form's solve, so the two
    agree to rounding."""
    from stda_b200.engine import Engine, Keywords, boundary_inputs
    mol, ints = benzene
    kw = Keywords(ax=0.5, e_thr_ev=10.0, solver=2)
    out = []
    for precision in (0, 1):
        eng = Engine(0, precision)          # no flag: the size gates apply
        eng.load(boundary_inputs(mol, ints))
        out.append(eng.polarizability(kw, [0.0, 0.05])[0])
        eng.close()
    assert np.abs(out[0] - out[1]).max() <= 1e-12 * np.abs(out[0]).max()


@pytest.mark.parametrize("precision", [0, 1])
def test_std_dft_iterative_vs_dense_oracle(precision):
    """sTD-DFT roots by the matrix-free subspace solver (solver 2) against the
    oracle's dense srpapack restatement: roots to 1e-9 Eh, f_L and f_V to 1e-5
    relative (FP64 products in both forms)."""
    from stda_b200 import synth
    mol, ints = synth.random_molecule(40, seed=4, with_ints=True)
    kw = dict(ax=0.5, e_thr_ev=8.0)
    eng, sol, iconf, ed = _run(mol, ints, precision=precision, rpa=True, nroots=10, solver=2,
                               conv_tol=1e-8, **kw)
    ref = _oracle(mol, ints, rpa=True, **kw)
    assert _same_csf(ref, iconf)
    n = min(10, len(ref.omega))
    assert len(sol.omega) == n
    assert np.abs(sol.omega - ref.omega[:n]).max() < 1e-9
    assert np.allclose(sol.fL, ref.fL[:n], rtol=1e-5, atol=1e-8)
    assert np.allclose(sol.fV, ref.fV[:n], rtol=1e-5, atol=1e-8)
    assert np.allclose(sol.RL, ref.RL[:n], rtol=1e-4, atol=1e-6)


def test_std_dft_iterative_pure_functional(benzene):
    """ax = 0: A-B is diagonal (rrpamat stda.f:1893-1928)."""
    mol, ints = benzene
    kw = dict(ax=0.0, e_thr_ev=10.0)
    eng, sol, iconf, ed = _run(mol, ints, rpa=True, nroots=8, solver=2, conv_tol=1e-8, **kw)
    ref = _oracle(mol, ints, rpa=True, **kw)
    assert np.abs(sol.omega - ref.omega[:8]).max() < 1e-9
    assert np.allclose(sol.fL, ref.fL[:8], rtol=1e-5, atol=1e-8)


def test_indefinite_overlap_is_refused(water):
    """makel stops on a negative overlap eigenvalue (stda.f:1658-1670); the
    engine's Newton-Schulz S^1/2 reports it as STD2G_ES_NOT_PD."""
    from stda_b200.engine import Engine, Keywords, Std2gError, boundary_inputs
    mol, ints = water
    b = boundary_inputs(mol, ints)
    S = b.S.copy()
    S[1] = 1.5            # element (2, 1): |S_21| > 1 makes S indefinite
    b.S = S
    eng = Engine(0, 0)
    eng.load(b)
    with pytest.raises(Std2gError) as e:
        eng.solve(Keywords(ax=1.0, e_thr_ev=20.0))
    assert e.value.name == "ES_NOT_PD"
    eng.close()


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("rpa", [False, True])
def test_dominant_csfs_and_error_estimates(water, precision, rpa):
    """The state table's three dominant CSFs per root (stda.f:1222-1358)
    against the oracle's restatement of the reference's selection, and the
    per-root error estimate: |w - w_FP64 exact| stays below err_est for every
    root that has one (Davidson and dense TDA)."""
    from oracle.stda_fp64 import dominant_csfs
    from stda_b200 import synth
    mol, ints = synth.random_molecule(28, seed=9, with_ints=True)
    kw = dict(ax=0.5, e_thr_ev=8.0, rpa=rpa)
    ref = _oracle(mol, ints, **kw)
    val, oi, oa = dominant_csfs(ref)
    for nroots, solver in ((0, 1), (8, 2)):
        eng, sol, iconf, ed = _run(mol, ints, precision, nroots=nroots, solver=solver,
                                   conv_tol=1e-8, **kw)
        eng.close()
        n = len(sol.omega)
        dom = sol.extras["dominant"]
        # the leading CSF of every root is the oracle's; the three weights agree
        # (the order of nearly equal second / third weights may differ)
        assert np.array_equal(dom["i"][:, 0], oi[:n, 0])
        assert np.array_equal(dom["a"][:, 0], oa[:n, 0])
        if rpa:
            assert np.allclose(dom["value"], val[:n], atol=1e-6)
        else:
            assert np.allclose(np.abs(dom["value"]), np.abs(val[:n]), atol=1e-6)
        err = sol.extras["err_est"]
        resid = sol.extras["resid"]
        if rpa and solver == 1:
            assert np.all(err == -1.0) and np.all(resid == -1.0)
        else:
            assert np.all(err >= 0.0) and np.all(resid >= 0.0)
            assert np.all(np.abs(sol.omega - ref.omega[:n]) <= err + 1e-12), (
                np.abs(sol.omega - ref.omega[:n]), err)

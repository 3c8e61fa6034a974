"""Quadratic-response consumers on the engine, through the C ABI.

beta(-2w; w, w) of sTD-DFT (lresp1, linear_response.f:196-700) is checked
against the reference's golden beta_HRS values (BETA_TEST1-3, water, at w = 0
and the two wavelengths of tests/wavelength; the reference's rule is 1e-3,
its real*4 solves sit ~1e-6 from FP64) and, tensor element by element,
against the FP64 oracle: 1e-8 relative to the largest element for the FP64
form and 1e-6 for the mixed form (its responses are refined to FP64
residuals below 1e-10).
"""
import json
import os

import numpy as np
import pytest

from oracle.stda_fp64 import Params, shg_hyperpolarizability, stda as oracle_stda
from tests.conftest import GOLDEN

pytestmark = pytest.mark.gpu

EXPECTED = json.load(open(os.path.join(GOLDEN, "reference_expected.json")))


def _wavelengths():
    with open(os.path.join(GOLDEN, "wavelength")) as fh:
        return [float(t) for t in fh.read().split()]


def _engine_beta(mol, ints, precision, wl, **kw):
    from stda_b200.engine import Engine, Keywords, boundary_inputs
    eng = Engine(0, precision)
    eng.load(boundary_inputs(mol, ints))
    out = eng.hyperpolarizability(Keywords(**kw), wl)
    eng.close()
    return out


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["BETA_TEST1", "BETA_TEST2", "BETA_TEST3"])
def test_beta_hrs_golden(water, name, precision):
    mol, ints = water
    case = EXPECTED[name]
    wl = _wavelengths()
    ev, beta, hrs = _engine_beta(mol, ints, precision, wl, **case["args"])
    exp = np.array(case["rows"])
    assert np.all(np.abs(ev - exp[:, 0]) <= 1e-6)
    assert np.all(np.abs(hrs - exp[:, 1]) <= 1e-3)     # the reference's rule
    assert np.all(np.abs(hrs - exp[:, 1]) <= 1e-5)     # FP64 vs its real*4 solves
    ref = oracle_stda(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), *ints,
                      Params(rpa=True, **case["args"]))
    _, bref, href = shg_hyperpolarizability(ref, wl)
    tol = 1e-8 if precision == 0 else 1e-6
    scale = np.abs(bref).max(axis=(1, 2, 3))
    assert np.all(np.abs(beta - bref).max(axis=(1, 2, 3)) <= tol * scale)
    assert np.allclose(hrs, href, rtol=tol)


def test_beta_benzene_both_forms():
    """A molecule with a richer tensor: both forms against the oracle."""
    from stda_b200 import synth
    mol, ints = synth.benzene(with_ints=True)
    kw = dict(ax=0.5, e_thr_ev=10.0)
    wl = [1064.0, 800.0]
    ref = oracle_stda(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), *ints,
                      Params(rpa=True, **kw))
    _, bref, href = shg_hyperpolarizability(ref, wl)
    scale = np.abs(bref).max(axis=(1, 2, 3))
    for precision, tol in ((0, 1e-8), (1, 1e-6)):
        ev, beta, hrs = _engine_beta(mol, ints, precision, wl, **kw)
        err = np.abs(beta - bref).max(axis=(1, 2, 3))
        assert np.all(err <= tol * scale), (precision, err / scale)
        assert np.allclose(hrs, href, rtol=tol)


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("name", ["2PA_TEST1", "2PA_TEST2", "2PA_TEST3"])
def test_two_photon_golden(water, name, precision):
    """-2PA 3 (lresp_2PA_SP): energies within 1e-3 eV, delta_par, delta_perp,
    delta_circ and rho within 1e-2 (the reference's rules; the goldens carry
    three decimals), and every entry against the FP64 oracle to 1e-8."""
    from oracle.stda_fp64 import two_photon_absorption
    from stda_b200.engine import Engine, Keywords, boundary_inputs
    mol, ints = water
    case = EXPECTED[name]
    exp = np.array(case["rows"])
    eng = Engine(0, precision)
    eng.load(boundary_inputs(mol, ints))
    got = eng.two_photon(Keywords(**case["args"]), len(exp))
    eng.close()
    assert got.shape == exp.shape
    assert np.array_equal(got[:, 0], exp[:, 0])
    assert np.all(np.abs(got[:, 1] - exp[:, 1]) <= 1e-3)
    assert np.all(np.abs(got[:, 2:] - exp[:, 2:]) <= 1e-2)
    ref = oracle_stda(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), *ints,
                      Params(rpa=True, **case["args"]))
    want = two_photon_absorption(ref, len(exp))
    assert np.allclose(got, want, rtol=1e-8, atol=1e-10)


def test_two_photon_too_many_states(water):
    from stda_b200.engine import Engine, Keywords, Std2gError, boundary_inputs
    mol, ints = water
    eng = Engine(0, 0)
    eng.load(boundary_inputs(mol, ints))
    with pytest.raises(Std2gError) as e:
        eng.two_photon(Keywords(ax=1.0, e_thr_ev=20.0), 500)
    assert e.value.name == "EINVAL"
    eng.close()

"""The package's ``tda.dat`` writer against the oracle's (``stda.f:2235-2265``,
``apbtrafo.f:100-130``) on the oracle's water solutions: identical text for the
velocity-corrected (VELO) and the plain (UV) variants, the E_thr row rule of the
UV variant, and the MMASS sum over the whole mass table of ``block.f``."""
from types import SimpleNamespace

import numpy as np
import pytest

from oracle.stda_fp64 import AMS, Params, stda, tda_dat_text
from stda_b200.tdadat import molecular_mass, tda_dat


def _solve(water, **kw):
    mol, (S, L, V, M) = water
    p = Params(**kw)
    return p, stda(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), S, L, V, M, p)


@pytest.mark.parametrize("kw", [dict(ax=0.5, e_thr_ev=30.0),
                                dict(ax=0.5, e_thr_ev=30.0, velcorr=False),
                                dict(ax=1.0, e_thr_ev=20.0, rpa=True)])
def test_writer_matches_oracle(water, kw):
    p, res = _solve(water, **kw)
    sol = SimpleNamespace(omega=res.omega, fL=res.fL, fV=res.fV, RL=res.RL, RV=res.RV,
                          xmolw=molecular_mass(water[0].xyz4()[3]))
    keys = SimpleNamespace(rpa=p.rpa, velcorr=p.velcorr, e_thr_ev=p.e_thr_ev)
    assert tda_dat(sol, keys) == tda_dat_text(res, p)


def test_uv_variant_drops_roots_above_threshold():
    sol = SimpleNamespace(omega=np.array([0.1, 0.2, 0.5]), fL=np.ones(3), fV=np.ones(3),
                          RL=np.zeros(3), RV=np.zeros(3), xmolw=18.0152)
    thr_ev = 0.3 * 27.211385050
    uv = tda_dat(sol, SimpleNamespace(rpa=True, velcorr=True, e_thr_ev=thr_ev)).splitlines()
    velo = tda_dat(sol, SimpleNamespace(rpa=False, velcorr=True, e_thr_ev=thr_ev)).splitlines()
    assert uv[1] == " UV" and velo[1] == " VELO"
    assert len(uv) == 13 + 2 and len(velo) == 13 + 3      # VELO keeps every root
    assert uv[-1] == "   2    5.4423     1.000000     1.000000     0.000000     0.000000"


def test_mass_table_covers_every_element_of_the_reference_table():
    for z in range(1, 108):
        assert molecular_mass([z]) == AMS[z - 1], z
    assert molecular_mass([35, 53, 1, 1]) == pytest.approx(79.904 + 126.9045 + 2 * 1.0079)
    assert molecular_mass([60]) == 0.0            # lanthanides carry no mass in the table

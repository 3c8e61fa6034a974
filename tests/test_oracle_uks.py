"""The UKS restatement of sutda (oracle.stda_uks) on the CPU.

There are no unrestricted goldens upstream.  The restatement is pinned by a
known answer instead: a closed-shell molecule given as an unrestricted
wavefunction (alpha = beta MOs, occupation 1 each) has the union of the
restricted singlet and triplet excitations when every CSF is in the space
(the UKS A matrix splits into the singlet and triplet combinations), with the
singlets' f_L, f_V and R of the restricted oracle (itself pinned to the
EXCI goldens) and zero f for the triplets.  TDA and sTD-DFT.
"""
import numpy as np
import pytest

from oracle.stda_fp64 import Params, stda, stda_uks


def _as_uks(mol):
    n = mol.C.shape[1]
    C2 = np.hstack([mol.C, mol.C])
    eps2 = np.concatenate([mol.eps, mol.eps])
    occ2 = np.concatenate([mol.occ / 2, mol.occ / 2])
    csp = np.concatenate([np.ones(n, dtype=int), np.full(n, 2)])
    return C2, eps2, occ2, csp


@pytest.mark.parametrize("rpa", [False, True])
def test_closed_shell_uks_is_singlets_and_triplets(water, rpa):
    mol, (S, L, V, M) = water
    kw = dict(ax=0.5, e_thr_ev=60.0, rpa=rpa)
    C2, eps2, occ2, csp = _as_uks(mol)
    u = stda_uks(mol.xyz4(), C2, eps2, occ2, csp, mol.iaoat(), S, L, V, M, Params(**kw))
    s1 = stda(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), S, L, V, M, Params(**kw))
    t1 = stda(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), S, L, V, M,
              Params(triplet=True, **kw))
    assert u.nex == s1.nex + t1.nex and u.new == 0
    union = np.sort(np.concatenate([s1.omega, t1.omega]))
    assert len(u.omega) == len(union)
    assert np.abs(u.omega - union).max() < 1e-12
    # singlet roots carry the restricted singlets' strengths, triplets none
    for w, fl, fv in zip(u.omega, u.fL, u.fV):
        ks = np.nonzero(np.abs(s1.omega - w) < 1e-9)[0]
        kt = np.nonzero(np.abs(t1.omega - w) < 1e-9)[0]
        assert len(ks) + len(kt) >= 1
        if len(ks) and not len(kt):
            assert abs(fl - s1.fL[ks[0]]) < 1e-10 and abs(fv - s1.fV[ks[0]]) < 1e-10
        if len(kt) and not len(ks):
            assert abs(fl) < 1e-12


def test_open_shell_uks_basic_structure():
    """A doublet: CSFs of both spins, alpha block first, PT selection and the
    SOMO shift under the K-shift keyword change the diagonal only where
    somo_shift says (sutda.f:2402-2422)."""
    from stda_b200 import synth
    from stda_b200.integrals import ao_integrals
    mol = synth.random_molecule(12, seed=4)
    S, L, V, M = ao_integrals(mol)
    nel = int(np.rint(np.sum(mol.occ)))
    C2, eps2, occ2, csp = synth.open_shell(mol, nel // 2 + 1, nel // 2 - 1 + nel % 2, seed=5,
                                           ints=(S, L, V, M))
    p = Params(ax=0.5, e_thr_ev=8.0, fthr_ev=11.0)
    u = stda_uks(mol.xyz4(), C2, eps2, occ2, csp, mol.iaoat(), S, L, V, M, p)
    spin = u.extras["spin"]
    assert (spin == 1).any() and (spin == 2).any()
    assert np.all(np.diff(spin) >= 0)                  # alpha block, then beta
    assert u.extras["nuhf"] == 2 - nel % 2
    pk = Params(ax=0.5, e_thr_ev=8.0, fthr_ev=11.0, kshift=True)
    uk = stda_uks(mol.xyz4(), C2, eps2, occ2, csp, mol.iaoat(), S, L, V, M, pk)
    assert len(uk.omega) > 0 and np.all(uk.omega > 0)
    assert np.all(np.isfinite(uk.fL))

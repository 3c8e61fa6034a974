"""UKS sTDA / sTD-DFT on the engine (std2g_set_spins) against the FP64
restatement of sutda (oracle.stda_uks): the CSF list in sutda's order (alpha
block, then beta; primaries by energy, PT-selected by candidate order), the
PT-lowered diagonal, roots, f and R, in both forms, TDA and sTD-DFT, with the
K-shift and SOMO shift, and the closed-shell known answer (singlets and
triplets of the restricted engine)."""
import numpy as np
import pytest

from oracle.stda_fp64 import Params, stda_uks

pytestmark = pytest.mark.gpu


def _engine(precision):
    from stda_b200.engine import Engine, FLAG_TENSOR_ALWAYS
    return Engine(0, precision, flags=FLAG_TENSOR_ALWAYS if precision == 1 else 0)


def _load(eng, mol, ints, C2, eps2, occ2, csp):
    from stda_b200.engine import boundary_inputs
    import copy
    m = copy.copy(mol)
    m.C, m.eps, m.occ = C2, eps2, occ2
    eng.load(boundary_inputs(m, ints))
    eng.set_spins(csp)


def _combined_iconf(ref):
    noa, nob = ref.extras["no"]
    nva, nvb = ref.extras["nv"]
    sp = ref.extras["spin"]
    i = np.where(sp == 1, ref.iconf[:, 0], noa + ref.iconf[:, 0])
    a = np.where(sp == 1, ref.iconf[:, 1], nva + ref.iconf[:, 1])
    return np.stack([i, a], axis=1)


def _open_shell_case(seed=6, natoms=26):
    from stda_b200 import synth
    mol, ints = synth.random_molecule(natoms, seed=seed, with_ints=True)
    nel = int(np.rint(np.sum(mol.occ)))
    C2, eps2, occ2, csp = synth.open_shell(mol, nel // 2 + 1, nel // 2 - 1 + nel % 2,
                                           seed=seed + 50, ints=ints)
    return mol, ints, C2, eps2, occ2, csp


@pytest.mark.parametrize("precision", [0, 1])
@pytest.mark.parametrize("rpa", [False, True])
@pytest.mark.parametrize("kshift", [False, True])
def test_uks_matches_oracle(precision, rpa, kshift):
    from stda_b200.engine import Keywords
    mol, ints, C2, eps2, occ2, csp = _open_shell_case()
    kw = dict(ax=0.5, e_thr_ev=7.5, fthr_ev=10.5, rpa=rpa, kshift=kshift)
    ref = stda_uks(mol.xyz4(), C2, eps2, occ2, csp, mol.iaoat(), *ints, Params(**kw))
    eng = _engine(precision)
    _load(eng, mol, ints, C2, eps2, occ2, csp)
    sol = eng.solve(Keywords(**kw))
    iconf, ed = eng.csf()
    eng.close()
    assert ref.new > 0 and (ref.extras["spin"] == 2).any()
    got = np.stack([iconf[:, 0] - 1, iconf[:, 1] - 1 - sol.no], axis=1)
    assert np.array_equal(got, _combined_iconf(ref))
    assert np.abs(ed - ref.ed).max() < (1e-10 if precision == 0 else 2e-7)
    n = len(ref.omega)
    assert len(sol.omega) == n
    tol = 1e-8 if precision == 0 else 4e-6
    assert np.abs(sol.omega - ref.omega).max() < tol
    big = ref.fL > 1e-3
    rtol = 1e-6 if precision == 0 else 1e-4
    assert np.allclose(sol.fL[big], ref.fL[big], rtol=rtol)
    assert np.allclose(sol.RV, ref.RV, rtol=max(rtol, 1e-5), atol=1e-6)


def test_closed_shell_uks_engine_is_singlets_and_triplets(water):
    from stda_b200.engine import Engine, Keywords, boundary_inputs
    mol, ints = water
    n = mol.C.shape[1]
    C2 = np.hstack([mol.C, mol.C])
    eps2 = np.concatenate([mol.eps, mol.eps])
    occ2 = np.concatenate([mol.occ / 2, mol.occ / 2])
    csp = np.concatenate([np.ones(n, dtype=np.int32), np.full(n, 2, dtype=np.int32)])
    kw = dict(ax=0.5, e_thr_ev=60.0)
    eng = Engine(0, 0)
    _load(eng, mol, ints, C2, eps2, occ2, csp)
    u = eng.solve(Keywords(**kw))
    eng.load(boundary_inputs(mol, ints))
    s1 = eng.solve(Keywords(**kw))
    t1 = eng.solve(Keywords(triplet=True, **kw))
    eng.close()
    union = np.sort(np.concatenate([s1.omega, t1.omega]))
    assert len(u.omega) == len(union)
    assert np.abs(u.omega - union).max() < 1e-10


def test_uks_refuses_restricted_only_paths(water):
    from stda_b200.engine import Keywords, Std2gError
    mol, ints = water
    n = mol.C.shape[1]
    C2 = np.hstack([mol.C, mol.C])
    eps2 = np.concatenate([mol.eps, mol.eps])
    occ2 = np.concatenate([mol.occ / 2, mol.occ / 2])
    csp = np.concatenate([np.ones(n, dtype=np.int32), np.full(n, 2, dtype=np.int32)])
    eng = _engine(0)
    _load(eng, mol, ints, C2, eps2, occ2, csp)
    for call in (lambda: eng.solve(Keywords(ax=0.5, e_thr_ev=20.0, triplet=True)),
                 lambda: eng.polarizability(Keywords(ax=0.5, e_thr_ev=20.0), [0.0])):
        with pytest.raises(Std2gError) as e:
            call()
        assert e.value.name == "EINVAL"
    with pytest.raises(Std2gError):
        eng.set_spins(np.full(2 * n, 3, dtype=np.int32))
    eng.close()

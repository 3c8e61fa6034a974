"""AO one-electron integrals on the device (std2g_ao_integrals,
std2g_load_prims) against the host Obara-Saika restatement
(stda_b200/integrals.py: S, -<a|r|b>, -<a|d/dr|b>, <a|r x d/dr|b> with the
conventions of libcint.f:19-352, 653-756 and intslvm.f:213-300).

Covered: every Cartesian type up to f (s, p, d and f shells added to water),
STO-3G benzene and a random cluster; a solve loaded from the primitive list
equals the solve loaded with the host integrals; bad primitive lists are
refused before any device work.
"""
import copy

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _with_df_shells(mol):
    """Water plus d and f polarisation shells on O and a d shell on H."""
    from stda_b200.molden import Shell
    m = copy.deepcopy(mol)
    o = int(np.argmax(m.Z))
    h = [k for k in range(m.ncent) if k != o][0]
    m.shells = list(m.shells) + [
        Shell(o, 2, np.array([1.8, 0.45]), np.array([0.6, 0.5])),
        Shell(o, 3, np.array([1.1]), np.array([1.0])),
        Shell(h, 2, np.array([0.9]), np.array([1.0])),
        Shell(h, 1, np.array([0.75, 0.2]), np.array([0.4, 0.7])),
    ]
    m.C = None
    return m


def _device_ints(eng, mol):
    from stda_b200.engine import primitives
    xyz4 = np.hstack([mol.xyz, mol.Z[:, None].astype(np.float64)])
    return eng.ao_integrals(xyz4, mol.nao, primitives(mol))


def _host_ints(mol):
    from stda_b200.integrals import ao_integrals, pack_lower
    S, L, V, M = ao_integrals(mol)
    return pack_lower(S), pack_lower(L), pack_lower(V), pack_lower(M)


@pytest.mark.parametrize("case", ["water_spdf", "benzene", "cluster"])
def test_ao_integrals_match_host(water, case):
    from stda_b200 import synth
    from stda_b200.engine import Engine
    if case == "water_spdf":
        mol = _with_df_shells(water[0])
    elif case == "benzene":
        mol = synth.benzene()
    else:
        mol = synth.random_molecule(40, seed=5)
    eng = Engine(0, 0)
    dev = _device_ints(eng, mol)
    eng.close()
    host = _host_ints(mol)
    for name, d, h in zip("SLVM", dev, host):
        scale = max(1.0, np.abs(h).max())
        err = np.abs(d - h).max()
        assert err <= 1e-12 * scale, (case, name, err)
    # diagonal of the overlap: every AO normalised to one
    S = dev[0]
    n = mol.nao
    diag = S[[i * (i + 1) // 2 + i for i in range(n)]]
    assert np.abs(diag - 1.0).max() < 1e-12


def test_load_prims_solve_equals_host_integrals():
    from stda_b200 import synth
    from stda_b200.engine import Engine, Keywords, boundary_inputs, primitives
    mol, ints = synth.random_molecule(30, seed=11, with_ints=True)
    kw = Keywords(ax=0.5, e_thr_ev=8.0, nroots=12)
    eng = Engine(0, 0)
    eng.load(boundary_inputs(mol, ints))
    ref = eng.solve(kw)
    xyz4 = np.hstack([mol.xyz, mol.Z[:, None].astype(np.float64)])
    eng.load_prims(xyz4, mol.C, mol.eps, mol.occ, primitives(mol))
    got = eng.solve(kw)
    eng.close()
    assert got.csf_hash == ref.csf_hash
    assert np.abs(got.omega - ref.omega).max() < 1e-11
    assert np.allclose(got.fL, ref.fL, rtol=1e-8, atol=1e-12)
    assert np.allclose(got.RV, ref.RV, rtol=1e-7, atol=1e-10)


def test_ao_integrals_reject_bad_primitives(water):
    from stda_b200.engine import Engine, Std2gError, primitives
    mol = water[0]
    pr = primitives(mol)
    xyz4 = np.hstack([mol.xyz, mol.Z[:, None].astype(np.float64)])
    eng = Engine(0, 0)
    for field, value in (("ipty", 21), ("ipao", mol.nao + 1), ("ipat", 0), ("exip", -1.0)):
        bad = copy.deepcopy(pr)
        getattr(bad, field)[0] = value
        with pytest.raises(Std2gError) as e:
            eng.ao_integrals(xyz4, mol.nao, bad)
        assert e.value.name == "EINVAL", field
    eng.close()

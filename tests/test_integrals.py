"""Host-side AO integrals: symmetry, normalisation and a finite-difference check."""
import copy

import numpy as np

from stda_b200.integrals import ao_integrals, pack_lower, unpack_lower


def test_overlap_normalised(water):
    mol, (S, L, V, M) = water
    assert np.allclose(np.diag(S), 1.0, atol=1e-12)
    assert np.allclose(S, S.T)
    assert np.linalg.eigvalsh(S).min() > 0


def test_antisymmetry(water):
    mol, (S, L, V, M) = water
    assert np.allclose(V, -np.transpose(V, (0, 2, 1)), atol=1e-14)
    assert np.allclose(M, -np.transpose(M, (0, 2, 1)), atol=1e-14)
    assert np.allclose(L, np.transpose(L, (0, 2, 1)))


def test_velocity_is_overlap_derivative(water):
    """V[a,b] = -<a|d/dx|b> = dS_ab/dB_x for b on the displaced atom."""
    mol, (S, L, V, M) = water
    iao = mol.iaoat()
    h = 1e-5
    for atom in range(mol.ncent):
        for d in range(3):
            m1 = copy.deepcopy(mol)
            m1.xyz[atom, d] += h
            m2 = copy.deepcopy(mol)
            m2.xyz[atom, d] -= h
            dS = (ao_integrals(m1)[0] - ao_integrals(m2)[0]) / (2 * h)
            mask = (iao[None, :] == atom) & (iao[:, None] != atom)
            assert np.abs((V[d] - dS)[mask]).max() < 1e-8


def test_dipole_origin_shift(water):
    """-<a|x|b> shifts by -dx*S when the molecule is translated by dx."""
    mol, (S, L, V, M) = water
    m1 = copy.deepcopy(mol)
    m1.xyz[:, 0] += 0.7
    S1, L1, V1, M1 = ao_integrals(m1)
    assert np.allclose(L1[0], L[0] - 0.7 * S, atol=1e-12)
    assert np.allclose(V1, V, atol=1e-12)


def test_pack_roundtrip(water):
    mol, (S, L, V, M) = water
    n = mol.nao
    assert np.allclose(unpack_lower(pack_lower(S), n), S)
    assert np.allclose(unpack_lower(pack_lower(V[1]), n, antisym=True), V[1])

"""The primitive list handed to the device integrals (std2g_ao_integrals):
types follow the reference's 20 Cartesian types (intpack.f90:1213-1218) and
every AO's coefficients are normalised (readbasmold.f:355-378 then
normalize.f:23-80), checked here on the host with the same-centre primitive
overlap pi^1.5 (2l-1)!!(2m-1)!!(2n-1)!! / (2^L (a+b)^(L+1.5))."""
import math

import numpy as np

from stda_b200.engine import _CART_TYPE, primitives
from stda_b200.molden import Shell


def _dfact(n):
    r = 1.0
    while n > 1:
        r *= n
        n -= 2
    return r


def test_primitive_types_and_normalisation(water):
    import copy
    mol = copy.deepcopy(water[0])
    o = int(np.argmax(mol.Z))
    mol.shells = list(mol.shells) + [Shell(o, 2, np.array([1.8, 0.45]), np.array([0.6, 0.5])),
                                     Shell(o, 3, np.array([1.1, 0.3]), np.array([0.7, 0.4]))]
    pr = primitives(mol)
    inv = {v: k for k, v in _CART_TYPE.items()}
    assert sorted(inv) == list(range(1, 21))
    assert pr.ipao.min() == 1 and pr.ipao.max() == mol.nao
    assert np.all(np.diff(pr.ipao) >= 0)
    iaoat = np.zeros(mol.nao, dtype=int)
    iaoat[pr.ipao - 1] = pr.ipat
    assert np.array_equal(iaoat, mol.iaoat() + 1)
    for a in range(1, mol.nao + 1):
        sel = pr.ipao == a
        types = set(pr.ipty[sel])
        assert len(types) == 1
        lx, ly, lz = inv[types.pop()]
        L = lx + ly + lz
        al, c = pr.exip[sel], pr.cxip[sel]
        pref = math.pi ** 1.5 * _dfact(2 * lx - 1) * _dfact(2 * ly - 1) * _dfact(2 * lz - 1) / 2 ** L
        s = pref * np.sum(np.outer(c, c) / (al[:, None] + al[None, :]) ** (L + 1.5))
        assert abs(s - 1.0) < 1e-12, (a, s)

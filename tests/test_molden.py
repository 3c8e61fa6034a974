"""The molden reader behind the boundary inputs (``readbasmold.f:217-740``
conventions): a write/read round trip, Angstrom input, ``sp`` shells, omitted
MO coefficients, and the inputs it refuses (spherical or open-shell files)."""
import os

import numpy as np
import pytest

from stda_b200.molden import BOHR_ANGSTROM, read_molden, write_molden
from tests.conftest import GOLDEN

WATER = os.path.join(GOLDEN, "water_sto3g.molden")


def test_round_trip(tmp_path):
    mol = read_molden(WATER)
    path = tmp_path / "w.molden"
    write_molden(mol, str(path), title="round trip")
    back = read_molden(str(path))
    assert np.array_equal(back.Z, mol.Z)
    assert np.allclose(back.xyz, mol.xyz, rtol=0, atol=1e-11)
    assert [(s.atom, s.l) for s in back.shells] == [(s.atom, s.l) for s in mol.shells]
    for a, b in zip(back.shells, mol.shells):
        assert np.allclose(a.exps, b.exps, rtol=1e-10) and np.allclose(a.coefs, b.coefs, rtol=1e-10)
    assert np.allclose(back.C, mol.C, rtol=1e-14, atol=1e-15)
    assert np.array_equal(back.eps, mol.eps) and np.array_equal(back.occ, mol.occ)
    assert back.nao == mol.nao == 7 and np.array_equal(back.iaoat(), mol.iaoat())


MINI = """[Molden Format]
[Atoms] {unit}
O     1    8 {x:.12f} 0.0 0.0
H     2    1 0.0 {y:.12f} 0.0
[GTO]
  1 0
 sp 2 1.00
  5.0 0.4 0.6
  1.0 0.7 0.5

  2 0
 s 1 1.00
  0.8 1.0

[MO]
 Sym= 1
 Ene= -0.5
 Spin= Alpha
 Occup= 2.0
    1 0.9
    5 0.1
 Sym= 1
 Ene= 0.3
 Spin= Alpha
 Occup= 0.0
    2 1.0D-01
"""


def test_angstrom_sp_shells_and_sparse_coefficients(tmp_path):
    p_ang = tmp_path / "a.molden"
    p_ang.write_text(MINI.format(unit="Angs", x=1.0, y=0.5))
    p_au = tmp_path / "b.molden"
    p_au.write_text(MINI.format(unit="AU", x=1.0 / BOHR_ANGSTROM, y=0.5 / BOHR_ANGSTROM))
    a, b = read_molden(str(p_ang)), read_molden(str(p_au))
    assert np.allclose(a.xyz, b.xyz, rtol=0, atol=1e-11)
    assert np.isclose(a.xyz[0, 0], 1.0 / BOHR_ANGSTROM)
    # the sp shell becomes an s and a p shell with shared exponents: 1 + 3 + 1 AOs
    assert [(s.atom, s.l) for s in a.shells] == [(0, 0), (0, 1), (1, 0)]
    assert np.array_equal(a.shells[0].exps, a.shells[1].exps)
    assert np.array_equal(a.shells[0].coefs, [0.4, 0.7]) and np.array_equal(a.shells[1].coefs, [0.6, 0.5])
    assert a.nao == 5 and list(a.iaoat()) == [0, 0, 0, 0, 1]
    # coefficients not listed are zero; Fortran D exponents are read
    assert np.allclose(a.C[:, 0], [0.9, 0, 0, 0, 0.1]) and np.allclose(a.C[:, 1], [0, 0.1, 0, 0, 0])
    assert np.array_equal(a.eps, [-0.5, 0.3]) and np.array_equal(a.occ, [2.0, 0.0])


def test_refuses_spherical_reads_open_shell(tmp_path):
    sph = tmp_path / "s.molden"
    sph.write_text(MINI.format(unit="AU", x=1.0, y=1.0).replace("[GTO]", "[5D]\n[GTO]"))
    with pytest.raises(ValueError, match="spherical"):
        read_molden(str(sph))
    uhf = tmp_path / "u.molden"
    uhf.write_text(MINI.format(unit="AU", x=1.0, y=1.0).replace(
        " Ene= 0.3\n Spin= Alpha", " Ene= 0.3\n Spin= Beta"))
    mol = read_molden(str(uhf))
    assert mol.csp is not None and list(mol.csp).count(2) == 1


def test_open_shell_molden_round_trip(tmp_path):
    """Spin= Beta MOs give Molecule.csp (the reference sends such files to
    sutda, main.f:933); a written open-shell file reads back unchanged."""
    import copy
    from stda_b200 import synth
    from stda_b200.molden import read_molden, write_molden
    mol = synth.random_molecule(8, seed=2)
    C2, eps2, occ2, csp = synth.open_shell(mol, 9, 8, seed=3)
    m = copy.deepcopy(mol)
    m.C, m.eps, m.occ, m.csp = C2, eps2, occ2, csp
    path = str(tmp_path / "uks.molden")
    write_molden(m, path)
    back = read_molden(path)
    assert back.csp is not None and np.array_equal(back.csp, csp)
    assert np.allclose(back.C, C2, atol=1e-13) and np.allclose(back.eps, eps2)
    assert np.array_equal(back.occ, occ2)

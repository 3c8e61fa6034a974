"""xTB input path (readxtb.f:38-200, -xtb defaults main.f:202-219).

CPU: the wfn.xtb record layout round-trips, damaged files are refused, the
keyword defaults are the reference's.  GPU: a wfn.xtb file read back and
loaded through std2g_load_prims (AO integrals formed on the device from its
primitive list) gives the FP64 oracle's CSF list and roots under the -xtb
keywords (ax 0.5, alpha 2, beta 4, K-shift on).
"""
import numpy as np
import pytest

from stda_b200.xtb import from_molecule, read_wfn_xtb, write_wfn_xtb, xtb_keywords


def _wf(seed=7, natoms=24):
    from stda_b200 import synth
    mol, ints = synth.random_molecule(natoms, seed=seed, with_ints=True)
    return mol, ints, from_molecule(mol)


def test_wfn_xtb_round_trip(tmp_path):
    mol, _, wf = _wf()
    p = str(tmp_path / "wfn.xtb")
    write_wfn_xtb(p, wf)
    got = read_wfn_xtb(p)
    assert got.imethod == 1 and got.nbf == mol.nao and got.ncent == mol.ncent
    assert np.array_equal(got.Z, wf.Z) and np.array_equal(got.xyz, wf.xyz)
    for f in ("ipty", "ipao", "ipat", "exip", "cxip"):
        assert np.array_equal(getattr(got.prims, f), getattr(wf.prims, f)), f
    assert np.array_equal(got.C, wf.C)
    assert np.array_equal(got.eps, wf.eps) and np.array_equal(got.occ, wf.occ)
    assert got.atnam[0] in ("C", "N", "O", "H")


def test_wfn_xtb_unrestricted_layout(tmp_path):
    _, _, wf = _wf(seed=3, natoms=12)
    wf.imethod = 2
    wf.C = np.stack([wf.C, wf.C[:, ::-1]])
    wf.eps = np.stack([wf.eps, wf.eps + 0.01])
    wf.occ = np.stack([wf.occ / 2, wf.occ / 2])
    p = str(tmp_path / "wfn.xtb")
    write_wfn_xtb(p, wf)
    got = read_wfn_xtb(p)
    assert got.imethod == 2 and got.C.shape == wf.C.shape
    assert np.array_equal(got.C, wf.C) and np.array_equal(got.eps, wf.eps)


def test_wfn_xtb_damaged_files_refused(tmp_path):
    _, _, wf = _wf(seed=5, natoms=10)
    p = str(tmp_path / "wfn.xtb")
    write_wfn_xtb(p, wf)
    raw = open(p, "rb").read()
    q = str(tmp_path / "cut.xtb")
    open(q, "wb").write(raw[:-12])
    with pytest.raises(ValueError):
        read_wfn_xtb(q)
    bad = bytearray(raw)
    bad[4:8] = (3).to_bytes(4, "little")        # imethod 3
    open(q, "wb").write(bytes(bad))
    with pytest.raises(ValueError):
        read_wfn_xtb(q)


def test_xtb_keyword_defaults():
    kw = xtb_keywords(e_thr_ev=8.0)
    assert (kw.ax, kw.alpha_k, kw.beta_j) == (0.5, 2.0, 4.0)
    assert kw.kshift and (kw.shftmax, kw.shftwidth, kw.shftsteep) == (0.5, 0.1, 4.0)
    assert kw.e_thr_ev == 8.0


@pytest.mark.gpu
@pytest.mark.parametrize("precision", [0, 1])
def test_xtb_path_matches_oracle(tmp_path, precision):
    from oracle.stda_fp64 import Params, stda as oracle_stda
    from stda_b200.engine import Engine
    from stda_b200.xtb import load_xtb
    mol, ints, wf = _wf(seed=21, natoms=36)
    p = str(tmp_path / "wfn.xtb")
    write_wfn_xtb(p, wf)
    kw = xtb_keywords(e_thr_ev=7.0, nroots=10, conv_tol=1e-9)
    eng = Engine(0, precision)
    load_xtb(eng, read_wfn_xtb(p))
    sol = eng.solve(kw)
    iconf, ed = eng.csf()
    eng.close()
    ref = oracle_stda(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), *ints,
                      Params(ax=0.5, e_thr_ev=7.0, alpha_k=2.0, beta_j=4.0, kshift=True))
    # same CSF list in the same order as the oracle
    got = np.stack([iconf[:, 0] - 1, iconf[:, 1] - 1 - ref.no], axis=1)
    assert got.shape == ref.iconf.shape and np.array_equal(got, ref.iconf)
    n = len(sol.omega)
    assert np.abs(sol.omega - ref.omega[:n]).max() < (1e-8 if precision == 0 else 4e-6)
    big = ref.fL[:n] > 1e-3
    assert np.allclose(sol.fL[big], ref.fL[:n][big], rtol=1e-4)


@pytest.mark.gpu
def test_xtb_unrestricted_path_matches_uks_oracle(tmp_path):
    """An unrestricted wfn.xtb (imethod 2) goes through the device integrals
    and the UKS path: the sutda restatement's CSFs and roots under -xtb."""
    from oracle.stda_fp64 import Params, stda_uks
    from stda_b200 import synth
    from stda_b200.engine import Engine
    from stda_b200.xtb import XtbWavefunction, load_xtb
    mol, ints = synth.random_molecule(20, seed=14, with_ints=True)
    nel = int(np.rint(np.sum(mol.occ)))
    C2, eps2, occ2, csp = synth.open_shell(mol, nel // 2 + 1, nel // 2 - 1 + nel % 2, seed=15,
                                           ints=ints)
    n = mol.nao
    base = from_molecule(mol)
    wf = XtbWavefunction(2, base.atnam, base.xyz, base.Z, n, base.prims,
                         np.stack([C2[:, :n], C2[:, n:]]), np.stack([eps2[:n], eps2[n:]]),
                         np.stack([occ2[:n], occ2[n:]]))
    p = str(tmp_path / "wfn.xtb")
    write_wfn_xtb(p, wf)
    kw = xtb_keywords(e_thr_ev=7.0, nroots=8, conv_tol=1e-9)
    eng = Engine(0, 0)
    load_xtb(eng, read_wfn_xtb(p))
    sol = eng.solve(kw)
    eng.close()
    ref = stda_uks(mol.xyz4(), C2, eps2, occ2, csp, mol.iaoat(), *ints,
                   Params(ax=0.5, e_thr_ev=7.0, alpha_k=2.0, beta_j=4.0, kshift=True))
    assert np.abs(sol.omega - ref.omega[:len(sol.omega)]).max() < 1e-8

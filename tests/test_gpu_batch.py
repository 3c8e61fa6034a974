"""Batched eigensolves across contexts (std2g_batch_*, server flag
STD2G_FLAG_BATCH_EIGEN): every molecule's result equals the unbatched solve's
and the FP64 oracle's.

The request server's slots hand their TDA eigenproblems to one lockstep
Davidson (batch_davidson.cuh).  Checked through the C ABI:
* a mix of molecules (different CSF counts and iteration counts) submitted at
  once: CSF lists identical to the unbatched engine's, roots within 1e-9 Eh,
  f_L per degenerate level within 1e-5 relative, and the batch really held
  several problems per iteration;
* one molecule against the FP64 oracle's dense diagonalisation (roots 1e-9 Eh,
  f_L 1e-5 relative), in both forms;
* contexts attached to a batch directly (std2g_attach_batch), solving on
  their own host threads at the same time, equal to the same contexts
  detached.
"""
import threading

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

KW = dict(ax=0.5, e_thr_ev=7.0, nroots=12, conv_tol=1e-7)


def _molecules():
    from stda_b200 import synth
    from stda_b200.engine import boundary_inputs
    out = []
    for natoms, seed in [(22, 31), (30, 32), (26, 33), (40, 34), (34, 35), (28, 36)]:
        mol, ints = synth.random_molecule(natoms, seed=seed, with_ints=True)
        out.append((mol, ints, boundary_inputs(mol, ints)))
    return out


def _levels(omega, f, gap=1e-5):
    """f summed over groups of roots closer than gap (degenerate levels)."""
    out, cur = [], f[0]
    for q in range(1, len(omega)):
        if omega[q] - omega[q - 1] < gap:
            cur += f[q]
        else:
            out.append(cur)
            cur = f[q]
    out.append(cur)
    return np.array(out)


def _close(a, b):
    assert a.csf_hash == b.csf_hash and a.nci == b.nci
    assert len(a.omega) == len(b.omega)
    assert np.abs(a.omega - b.omega).max() < 1e-9
    la, lb = _levels(b.omega, a.fL), _levels(b.omega, b.fL)
    assert np.allclose(la, lb, rtol=1e-5, atol=1e-9)


def _alone(mols, precision):
    from stda_b200.engine import Engine, Keywords
    out = []
    for _, _, b in mols:
        eng = Engine(0, precision)
        eng.load(b)
        out.append(eng.solve(Keywords(**KW)))
        eng.close()
    return out


@pytest.mark.parametrize("precision", [1, 0])
def test_batched_server_same_as_alone(precision):
    from stda_b200.engine import FLAG_BATCH_EIGEN, Keywords, Server
    mols = _molecules()
    alone = _alone(mols, precision)
    assert all(320 < s.nci <= 6144 for s in alone)   # every problem is batch-eligible
    srv = Server(0, precision, slots=len(mols), flags=FLAG_BATCH_EIGEN)
    tickets = [srv.submit(b, Keywords(**KW)) for _, _, b in mols]
    res = [srv.wait(t) for t in tickets]
    bst = srv.batch_stats()
    srv.close()
    for (sol, _, _, _), ref in zip(res, alone):
        _close(sol, ref)
    assert bst["problems"] == len(mols)
    assert bst["mean_batch"] > 1.5        # several problems per batched iteration


@pytest.mark.parametrize("precision", [1, 0])
def test_batched_vs_oracle(precision):
    from oracle.stda_fp64 import Params as OParams, stda as oracle_stda
    from stda_b200.engine import FLAG_BATCH_EIGEN, Keywords, Server
    mol, ints, b = _molecules()[1]
    srv = Server(0, precision, slots=2, flags=FLAG_BATCH_EIGEN)
    sol = srv.wait(srv.submit(b, Keywords(**KW)))[0]
    srv.close()
    S, L, V, M = ints
    kw = {k: v for k, v in KW.items() if k not in ("nroots", "conv_tol")}
    ref = oracle_stda(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), S, L, V, M,
                      OParams(**kw))
    n = len(sol.omega)
    assert n == KW["nroots"] and len(ref.omega) >= n
    assert np.abs(sol.omega - ref.omega[:n]).max() < 1e-9
    assert np.allclose(_levels(ref.omega[:n], sol.fL), _levels(ref.omega[:n], ref.fL[:n]),
                       rtol=1e-5, atol=1e-9)


def test_attached_contexts_on_threads():
    import ctypes as C
    from stda_b200.engine import Engine, Keywords, _check, library
    lib = library()
    mols = _molecules()[:4]
    engines = [Engine(0, 1) for _ in mols]
    for eng, (_, _, b) in zip(engines, mols):
        eng.load(b)
    detached = [eng.solve(Keywords(**KW)) for eng in engines]
    batch = C.c_void_p()
    _check(lib.std2g_batch_create(0, C.byref(batch)))
    for eng in engines:
        _check(lib.std2g_attach_batch(eng.ctx, batch))
    out = [None] * len(engines)
    errs = []

    def run(q):
        try:
            out[q] = engines[q].solve(Keywords(**KW))
        except Exception as e:   # reported below
            errs.append(e)

    th = [threading.Thread(target=run, args=(q,)) for q in range(len(engines))]
    for t in th:
        t.start()
    for t in th:
        t.join()
    assert not errs
    assert all(lib.std2g_last_batched(eng.ctx) == 1 for eng in engines)
    pr, it, mem = C.c_int64(), C.c_int64(), C.c_int64()
    _check(lib.std2g_batch_stats(batch, C.byref(pr), C.byref(it), C.byref(mem), None))
    for eng in engines:
        _check(lib.std2g_attach_batch(eng.ctx, None))
        eng.close()
    lib.std2g_batch_destroy(batch)
    for a, b in zip(out, detached):
        _close(a, b)
    assert pr.value == len(engines) and mem.value > it.value

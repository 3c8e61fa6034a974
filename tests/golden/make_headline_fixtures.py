"""Oracle fixtures for the benchmark-sized molecules (TEST INFRASTRUCTURE).

Runs the FP64 oracle (``oracle/stda_fp64.py``) on the synthetic molecules of
the benchmark and writes what the GPU tests compare the engine against:

* ``flake8_pt.npz``   C384H48 flake (1584 AOs), ax 0.5, E_thr 7 eV, thrp 1e-4:
  window sizes, primary / candidate / PT-selected counts, the selected CSF
  list (i, a) in order and the diagonal after PT lowering (``ptselect``,
  ``stda.f:1773-1863``).  No A matrix (it would not fit the oracle).
* ``flake3_roots.npz`` C54H18 flake, same keywords: the CSF list, the lowest
  50 roots of the dense A and their f_L, f_V, R_L, R_V (velocity-corrected,
  ``apbtrafo.f:23-300``).
* ``chain200_alpha.npz`` 200-atom C/N/O/H chain, ax 0.5, E_thr 7 eV:
  alpha(omega) at omega = 0, 0.03, 0.06, 0.09, 0.12 Eh (``lresp``,
  ``linear_response.f:23-192``) from the dense A+B, A-B.

The molecules come from ``stda_b200.synth`` (seeded), the same generator the
tests and ``bench.py`` use on the GPU box, so the fixtures need no reference
checkout.  Runtime on 8 host cores: ~10-20 minutes, most of it the flake-8 PT
selection and the chain's dense solves.

Usage: python tests/golden/make_headline_fixtures.py [flake8|flake3|chain|all]
"""
import os
import sys
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.stda_fp64 import Params, dynamic_polarizability, stda  # noqa: E402
from stda_b200 import synth  # noqa: E402

KW = dict(ax=0.5, e_thr_ev=7.0, thrp=1e-4)
CHAIN_OMEGA = [0.0, 0.03, 0.06, 0.09, 0.12]


def fnv1a(iconf):
    """FNV-1a over the (i, a) int32 pairs, as std2g_result.csf_hash."""
    h = 1469598103934665603
    for b in np.ascontiguousarray(iconf.astype(np.int32)).tobytes():
        h ^= b
        h = (h * 1099511628211) & 0xFFFFFFFFFFFFFFFF
    return h


def _oracle(mol, ints, **kw):
    S, L, V, M = ints
    return lambda p, **x: stda(mol.xyz4(), mol.C, mol.eps, mol.occ, mol.iaoat(), S, L, V, M, p,
                               **x)


def flake8():
    t0 = time.time()
    mol, ints = synth.graphene_flake(8, with_ints=True)
    res = _oracle(mol, ints)(Params(**KW), want_A=False)
    np.savez_compressed(
        os.path.join(HERE, "flake8_pt.npz"), no=res.no, nv=res.nv, nex=res.nex,
        nexpt=res.nexpt, new=res.new, iconf=res.iconf.astype(np.int16), ed=res.ed,
        csf_hash=np.uint64(fnv1a(res.iconf)))
    print(f"flake8: nex {res.nex} nexpt {res.nexpt} new {res.new} nci {len(res.iconf)} "
          f"({time.time() - t0:.0f} s)", flush=True)


def flake3(nroots=50):
    t0 = time.time()
    mol, ints = synth.graphene_flake(3, with_ints=True)
    res = _oracle(mol, ints)(Params(**KW))
    k = min(nroots, len(res.omega))
    np.savez_compressed(
        os.path.join(HERE, "flake3_roots.npz"), nex=res.nex, nexpt=res.nexpt, new=res.new,
        iconf=res.iconf.astype(np.int16), ed=res.ed, csf_hash=np.uint64(fnv1a(res.iconf)),
        omega=res.omega[:k], fL=res.fL[:k], fV=res.fV[:k], RL=res.RL[:k], RV=res.RV[:k])
    print(f"flake3: nci {len(res.iconf)} roots {len(res.omega)} ({time.time() - t0:.0f} s)",
          flush=True)


def chain():
    t0 = time.time()
    mol, ints = synth.chain(200, with_ints=True)
    res = _oracle(mol, ints)(Params(rpa=True, **KW), want_roots=False)
    alpha = dynamic_polarizability(res, CHAIN_OMEGA)
    np.savez_compressed(
        os.path.join(HERE, "chain200_alpha.npz"), nci=len(res.iconf),
        csf_hash=np.uint64(fnv1a(res.iconf)), omega=np.array(CHAIN_OMEGA), alpha=alpha)
    print(f"chain: nci {len(res.iconf)} ({time.time() - t0:.0f} s)", flush=True)


if __name__ == "__main__":
    what = sys.argv[1] if len(sys.argv) > 1 else "all"
    for name, fn in (("flake3", flake3), ("chain", chain), ("flake8", flake8)):
        if what in (name, "all"):
            fn()

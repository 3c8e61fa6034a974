"""The engine's FP64 matrix product (dgemm.cuh: DMMA m8n8k4 tiles with a
deterministic split-K), through std2g_dgemm_check, against numpy.

Shapes cover ragged edges (not multiples of the 64 x 64 x 16 tile), k = 0
(C = beta C), every op(A) / op(B) combination, batched members, beta = 0
with NaN in C (C must not be read) and the tall-skinny Davidson shapes that
take the split-K path; split-K results are bit-identical from run to run.
"""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _ref(A, B, Cm, ta, tb, alpha, beta):
    a = A.T if ta else A
    b = B.T if tb else B
    return alpha * (a @ b) + (beta * Cm if beta != 0 else 0.0)


def _operands(rng, m, n, k, ta, tb, batch=None):
    sa = (k, m) if ta else (m, k)
    sb = (n, k) if tb else (k, n)
    pre = () if batch is None else (batch,)
    return (rng.standard_normal(pre + sa), rng.standard_normal(pre + sb),
            rng.standard_normal(pre + (m, n)))


@pytest.mark.parametrize("ta", [False, True])
@pytest.mark.parametrize("tb", [False, True])
@pytest.mark.parametrize("mnk", [(1, 1, 1), (65, 63, 17), (128, 64, 48), (37, 200, 129),
                                 (300, 75, 20011), (9, 9, 70000)])
def test_dgemm_matches_numpy(ta, tb, mnk):
    from stda_b200.engine import dgemm_check
    rng = np.random.default_rng(hash((ta, tb) + mnk) % 2**32)
    m, n, k = mnk
    A, B, Cm = _operands(rng, m, n, k, ta, tb)
    got, _ = dgemm_check(A, B, Cm, ta, tb, alpha=-0.75, beta=0.5)
    ref = _ref(A, B, Cm, ta, tb, -0.75, 0.5)
    tol = 1e-14 * np.sqrt(k) * 8 + 1e-15
    assert np.abs(got - ref).max() <= tol * max(1.0, np.sqrt(k)), np.abs(got - ref).max()


def test_dgemm_k0_beta0_batch_and_determinism():
    from stda_b200.engine import dgemm_check
    rng = np.random.default_rng(3)
    # k = 0: C = beta C
    A, B, Cm = _operands(rng, 20, 30, 0, False, False)
    got, _ = dgemm_check(A, B, Cm, beta=2.0)
    assert np.array_equal(got, 2.0 * Cm)
    # beta = 0: NaN in C is not read
    A, B, Cm = _operands(rng, 70, 33, 40, True, False)
    Cm[:] = np.nan
    got, _ = dgemm_check(A, B, Cm, ta=True, beta=0.0)
    assert np.isfinite(got).all()
    assert np.abs(got - A.T @ B).max() < 1e-12
    # batched members, strided one after another
    A, B, Cm = _operands(rng, 50, 40, 90, False, True, batch=3)
    got, _ = dgemm_check(A, B, Cm, tb=True, alpha=1.0, beta=1.0)
    ref = np.stack([A[q] @ B[q].T + Cm[q] for q in range(3)])
    assert np.abs(got - ref).max() < 1e-12
    # split-K: the same bits twice
    A, B, Cm = _operands(rng, 300, 75, 40000, True, False)
    g1, _ = dgemm_check(A, B, Cm, ta=True)
    g2, _ = dgemm_check(A, B, Cm, ta=True)
    assert np.array_equal(g1, g2)
    assert np.abs(g1 - A.T @ B).max() < 1e-11


def test_gemm_stats_own_and_library_count_the_same_products():
    """std2g_gemm_stats: the FP64 products of a solve, counted with their
    algorithmic FLOPs; event timing only when switched on; the library
    baseline (cuBLAS) is counted the same way."""
    from stda_b200 import synth
    from stda_b200.engine import FLAG_LIBRARY_FP64, Engine, Keywords, boundary_inputs
    mol, ints = synth.benzene(with_ints=True)
    b = boundary_inputs(mol, ints)
    kw = Keywords(ax=0.5, e_thr_ev=10.0, nroots=4)
    st = {}
    for name, flags in (("own", 0), ("lib", FLAG_LIBRARY_FP64)):
        eng = Engine(0, 0, flags=flags)
        eng.load(b)
        eng.solve(kw)
        first = eng.gemm_stats()   # includes the S^1/2 products (once per load)
        eng.solve(kw)
        off = eng.gemm_stats()
        assert first["calls"] > off["calls"]
        assert off["calls"] > 0 and off["flop"] > 0 and off["ms"] == 0.0
        eng.set_gemm_timing(True)
        eng.solve(kw)
        st[name] = eng.gemm_stats()
        assert st[name]["ms"] > 0.0
        assert st[name]["calls"] == off["calls"] and st[name]["flop"] == off["flop"]
        eng.set_gemm_timing(False)
        eng.solve(kw)
        assert eng.gemm_stats()["ms"] == 0.0
        eng.close()
    # the two forms may take a different number of Davidson iterations (their
    # rounding differs), so only the setup products are compared loosely
    assert abs(st["own"]["flop"] - st["lib"]["flop"]) <= 0.5 * st["own"]["flop"]

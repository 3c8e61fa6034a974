"""The symmetric eigensolver of the Davidson Rayleigh-Ritz step
against cuSOLVER syevd: eigenvalues to 1e-11 relative, residuals
||A z - w z|| and orthogonality ||Z^T Z - I|| to 1e-10, including exactly
degenerate and tightly clustered spectra."""
import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _check(A, k):
    from stda_b200.engine import symeig_check
    w, Z, wr = symeig_check(A, k)
    scale = max(1.0, np.abs(wr).max())
    assert np.abs(w - wr[:k]).max() <= 1e-11 * scale, np.abs(w - wr[:k]).max()
    res = np.abs(A @ Z - Z * w[None, :]).max()
    assert res <= 1e-10 * scale, res
    orth = np.abs(Z.T @ Z - np.eye(k)).max()
    assert orth <= 1e-10, orth


def _random_sym(n, seed):
    rng = np.random.default_rng(seed)
    M = rng.standard_normal((n, n))
    return 0.5 * (M + M.T)


@pytest.mark.parametrize("n,k", [(1, 1), (2, 2), (5, 3), (37, 37), (75, 75), (120, 30),
                                 (200, 75), (224, 75), (300, 75), (320, 80), (320, 320)])
def test_random(n, k):
    _check(_random_sym(n, n), k)


def _with_spectrum(lam, seed):
    n = len(lam)
    rng = np.random.default_rng(seed)
    Q, _ = np.linalg.qr(rng.standard_normal((n, n)))
    return (Q * np.asarray(lam)[None, :]) @ Q.T


def test_degenerate_pairs_and_clusters():
    n = 150
    lam = np.sort(np.concatenate([np.repeat(np.linspace(0.1, 1.0, 40), 2),
                                  1.5 + 1e-10 * np.arange(10), np.linspace(2, 5, 60)]))
    A = _with_spectrum(lam, 3)
    A = 0.5 * (A + A.T)
    _check(A, 75)
    _check(A, n)
    lam2 = np.concatenate([np.full(6, 0.3), np.linspace(0.5, 2.0, 94)])   # a 6-fold eigenvalue
    A2 = _with_spectrum(lam2, 4)
    _check(0.5 * (A2 + A2.T), 20)


def test_davidson_like():
    # diag(theta) (previous Ritz values) bordered by new coupling columns
    rng = np.random.default_rng(7)
    k, nb = 75, 75
    n = k + nb
    A = np.zeros((n, n))
    A[:k, :k] = np.diag(np.sort(rng.uniform(0.2, 0.4, k)))
    B = 1e-4 * rng.standard_normal((k, nb))
    C = rng.standard_normal((nb, nb)) * 1e-3
    A[:k, k:] = B
    A[k:, :k] = B.T
    A[k:, k:] = 0.5 * (C + C.T) + np.diag(rng.uniform(0.3, 0.6, nb))
    _check(A, 75)

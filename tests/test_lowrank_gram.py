"""The low-rank form of the multimode pair contraction (CPU, numpy).

The library factors the overlap Gram matrix Γ[p][q] = γ_ijkl over the pairs
p = (i <= j), q = (k <= l) as Σ_k λ_k Q_k Q_kᵀ (eigenvalues above 1e-12 of
the largest) and contracts G[ij][q] = w_q Γ[p][q] (w_q = 2 for k < l) as
Σ_k U[p][k] Z_k, U = Q Λ, Z_k = Σ_q w_q Q[q][k] X_q.  These tests pin the
ranks of the Hermite-Gauss bases the configs use and the identity itself, on
the overlap tensor that problem.multimode_problem builds (the normalised
4-overlap integrals S_plmn of the HG profiles).
"""
import numpy as np
import pytest

from fiberlab_gpu import problem as P


def _gram(gamma, M):
    pairs = [(k, l) for k in range(M) for l in range(k, M)]
    gam = np.array([[gamma[i, j, k, l] for (k, l) in pairs] for (i, j) in pairs])
    w = np.array([1.0 if k == l else 2.0 for (k, l) in pairs])
    return gam, w


def _rank(gam):
    ev = np.abs(np.linalg.eigvalsh(gam))
    return int(np.sum(ev > 1e-12 * ev.max()))


@pytest.mark.parametrize("order,M,rank", [(2, 6, 15), (3, 10, 28), (3, 8, 22), (3, 7, 19),
                                          (3, 9, 25)])
def test_gram_rank_of_hermite_gauss_bases(order, M, rank):
    # products of two HG modes of total order <= 2n are a Gaussian times the
    # monomials of degree <= 2n: 15 (n = 1) or 28 (n = 3) of them
    fp = P.multimode_problem(order, 32, 256, 5.0, 0.3, 2e-9, 200e-15, 0,
                             raman_threshold_thz=-5.0)
    gam, _ = _gram(fp.gamma[:M, :M, :M, :M], M)
    assert np.allclose(gam, gam.T, rtol=0, atol=1e-12 * np.abs(gam).max())
    assert _rank(gam) == rank


def test_low_rank_contraction_identity():
    fp = P.multimode_problem(3, 32, 256, 5.0, 0.3, 2e-9, 200e-15, 0, raman_threshold_thz=-5.0)
    M = fp.M
    gam, w = _gram(fp.gamma, M)
    lam, Q = np.linalg.eigh(gam)
    keep = np.abs(lam) > 1e-12 * np.abs(lam).max()
    U = Q[:, keep] * lam[keep]
    V = w[:, None] * Q[:, keep]
    G = gam * w[None, :]
    X = np.random.default_rng(5).standard_normal((G.shape[1], 64))  # 64 time points
    full = G @ X
    low = U @ (V.T @ X)
    assert np.max(np.abs(full - low)) <= 1e-12 * np.max(np.abs(full))
    # the Raman convolution commutes with the sum over pairs: convolving the
    # rank sequences V^T X and contracting with U equals contracting first
    h = np.random.default_rng(6).standard_normal(64)
    conv = lambda A: np.real(np.fft.ifft(np.fft.fft(A, axis=1) * np.fft.fft(h)[None, :], axis=1))
    assert np.allclose(U @ conv(V.T @ X), conv(full), rtol=0, atol=1e-11 * np.abs(conv(full)).max())

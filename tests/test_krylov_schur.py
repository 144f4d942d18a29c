"""CPU tests of the Krylov-Schur eigen-solver that drives the Eliashberg eigenproblem."""

import numpy as np
import torch

from dgamore_b200.eliashberg_solver import krylov_schur


def _check(A, k, tol=1e-12):
    a = torch.as_tensor(A)
    v0 = torch.as_tensor(np.random.default_rng(3).random(A.shape[0]) + 0j)
    vals, vecs, status = krylov_schur(lambda x: a @ x, v0, k, tol, ncv=2 * k + 8)
    ref = np.linalg.eigvals(A)
    ref = ref[np.argsort(-ref.real)][:k]
    assert status == 0
    assert np.allclose(vals, ref.real, rtol=1e-9, atol=1e-10)
    for lam, v in zip(vals, vecs):
        r = A @ v - (v.conj() @ A @ v) / (v.conj() @ v) * v
        assert np.linalg.norm(r) < 1e-7 * max(1.0, abs(lam))


def test_hermitian_matrix_leading_eigenvalues():
    rng = np.random.default_rng(0)
    x = rng.standard_normal((300, 300)) + 1j * rng.standard_normal((300, 300))
    _check((x + x.conj().T) / 2, 4)


def test_non_hermitian_matrix_largest_real_parts():
    rng = np.random.default_rng(1)
    x = rng.standard_normal((200, 200)) + 1j * rng.standard_normal((200, 200))
    d = np.diag(np.linspace(0, 30, 200))
    _check(d + 0.3 * x, 4)


def test_small_operator_exhausts_the_space():
    rng = np.random.default_rng(2)
    x = rng.standard_normal((6, 6)) + 0j
    _check(x + x.T, 3)

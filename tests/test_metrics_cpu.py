"""The variable-size backward-error helper that gates the Cholesky bench (run here on
CPU tensors) agrees with the per-instance numpy definition."""
import numpy as np

from magma_b200 import testing as T


def test_backward_error_vbatched_matches_numpy():
    import torch

    rng = np.random.default_rng(0)
    ns = np.array([5, 1, 9, 5, 3, 9])
    nr = np.array([2, 1, 3, 1, 4, 2])
    offA = np.concatenate([[0], np.cumsum(ns * ns)[:-1]])
    offB = np.concatenate([[0], np.cumsum(ns * nr)[:-1]])
    A = rng.standard_normal(int((ns * ns).sum()))
    X = rng.standard_normal(int((ns * nr).sum()))
    B = rng.standard_normal(int((ns * nr).sum()))
    got = T.backward_error_vbatched_torch(torch.from_numpy(A), torch.from_numpy(X), torch.from_numpy(B),
                                          ns, nr, offA, offB).numpy()
    for i, (n, r) in enumerate(zip(ns, nr)):
        Ai = A[offA[i]:offA[i] + n * n].reshape(1, n, n)            # (batch, n, lda) column-major
        Xi = X[offB[i]:offB[i] + n * r].reshape(1, r, n)
        Bi = B[offB[i]:offB[i] + n * r].reshape(1, r, n)
        want = T.backward_error(Ai, Xi, Bi, n).max()
        assert abs(got[i] - want) <= 1e-12 * want, (i, got[i], want)

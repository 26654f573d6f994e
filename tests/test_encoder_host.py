"""Host-side pieces of the amortised-encoder experiment (no GPU): the input-gene selection from
the CSR counts against a dense restatement, and the Procrustes-aligned RMSE used to score
latent positions."""
import numpy as np

from gaspacho2_b200 import encoder, synth


def test_select_genes_matches_dense_variance():
    ds = synth.make(1, 5, N=400, G=60, init=False)
    y = ds.y
    dense = np.zeros((y.N, y.J))
    for j in range(y.J):
        dense[y.i[y.p[j]:y.p[j + 1]], j] = y.x[y.p[j]:y.p[j + 1]]
    v = np.log1p(dense / ds.ls[:, None])
    var = v.var(axis=0)
    want = np.sort(np.argsort(-var, kind="stable")[:17])
    got = encoder.select_genes(y, ds.ls, 17)
    assert got.dtype == np.int32 and np.array_equal(got, want)


def test_procrustes_rmse_invariances():
    rng = np.random.default_rng(0)
    B = rng.standard_normal((200, 4))
    Q, _ = np.linalg.qr(rng.standard_normal((4, 4)))
    A = 2.5 * B @ Q.T + rng.standard_normal(4)  # B rotated, scaled and shifted
    assert encoder.procrustes_rmse(A, B) < 1e-12
    C = rng.standard_normal((200, 4))
    assert encoder.procrustes_rmse(C, B) > 0.5

"""The start of a fit computed on the GPU (gpl_init_latent): the principal component scores of
log1p(y / s) against a dense SVD of the same centred matrix on the host, component by component
up to the sign; the k-means centres against Lloyd's algorithm on the host from the GPU's scores;
and the CLI's --init-latent writing Xi.bin and fitting from it."""
import os
import subprocess

import numpy as np
import pytest

from gaspacho2_b200 import GPLVM, synth
from gaspacho2_b200.formats import write_dataset

pytestmark = pytest.mark.gpu


def _host_scores(y, ls, Q):
    N, J = y.N, y.J
    D = np.zeros((N, J))
    for j in range(J):
        b, e = int(y.p[j]), int(y.p[j + 1])
        D[y.i[b:e], j] = np.log1p(y.x[b:e] / ls[y.i[b:e]])
    D -= D.mean(0)
    U, S, _ = np.linalg.svd(D, full_matrices=False)
    sc = U[:, :Q] * S[:Q]
    return (sc - sc.mean(0)) / sc.std(0), S


def test_pca_scores_match_host_svd():
    ds = synth.make(1, 3, N=1500, G=300, M=20, Q=5)
    ref, S = _host_scores(ds.y, ds.ls, ds.Q)
    with GPLVM.from_dataset(ds) as m:
        X, T = m.init_latent(pca_iters=200, kmeans_iters=25, seed=1)
    assert X.shape == (ds.N, ds.Q) and T.shape == (ds.M, ds.Q)
    gaps = S[:ds.Q] / S[1:ds.Q + 1]
    for q in range(ds.Q):
        r = abs(np.corrcoef(X[:, q], ref[:, q])[0, 1])
        print(f"component {q}: |corr| {r:.8f} (singular value gap {gaps[q]:.3f})")
        if gaps[q] > 1.02:  # a well separated component is determined up to sign
            assert r > 1 - 1e-6, (q, r)
    assert np.allclose(X.mean(0), 0, atol=1e-10) and np.allclose(X.std(0), 1, atol=1e-10)


def test_kmeans_centres_are_a_lloyd_fixed_point_quality():
    ds = synth.make(0, 4, N=2000, G=200, M=16, Q=2)
    with GPLVM.from_dataset(ds) as m:
        X, T = m.init_latent(pca_iters=100, kmeans_iters=40, seed=2)
    d = ((X[:, None, :] - T[None, :, :]) ** 2).sum(-1)
    lab = d.argmin(1)
    sse = d.min(1).sum()
    # each centre is the mean of the cells nearest to it (up to the last assignment step)
    for k in range(ds.M):
        if (lab == k).any():
            assert np.allclose(T[k], X[lab == k].mean(0), atol=5e-2)
    host = synth._kmeans(X, ds.M, np.random.default_rng(0), iters=40)
    sse_host = ((X[:, None, :] - host[None, :, :]) ** 2).sum(-1).min(1).sum()
    print(f"k-means within-cluster sum of squares: GPU {sse:.3f}, host Lloyd {sse_host:.3f}")
    assert sse <= 1.15 * sse_host


def test_cli_init_latent_writes_xi_and_fits(tmp_path, root):
    ds = synth.make(0, 5, N=800, G=100, M=10, Q=2)
    paths = write_dataset(str(tmp_path), ds.y, ds.z, ds.ls, ds.X0)
    os.remove(paths["Xi"])
    exe = os.path.join(root, "gaspacho2_b200", "bin", "ggplvm")
    r = subprocess.run([exe, paths["Y"], paths["Z"], paths["ls"], paths["Xi"], "-M", "10", "-Q", "2", "--init-latent",
                        "--max-outer", "1", "--max-lbfgs-iters", "3", "--out-dir", str(tmp_path), "--quiet"],
                       capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    Xi = np.fromfile(paths["Xi"], np.float64)
    assert Xi.shape[0] == ds.N * ds.Q and np.all(np.isfinite(Xi))
    T = np.fromfile(os.path.join(str(tmp_path), "Tau.bin"), np.float64)
    assert T.shape[0] == ds.M * ds.Q and np.all(np.isfinite(T))
    assert os.path.exists(os.path.join(str(tmp_path), "params.bin"))

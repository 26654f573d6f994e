"""The amortised encoder and the per-cell placement on the GPU.

* The encoder's loss and every parameter gradient of one training batch (tcgen05 BF16 products,
  FP32 accumulation) against the CPU oracle's float64 restatement with the same BF16 rounding
  points (oracle/encoder_oracle.py): loss within 1e-5 relative, each gradient within 2e-3 relative
  (L2), the FP32 accumulation order being the only difference.
* Training lowers the loss and the trained network predicts the latent coordinates of unseen
  cells.
* The per-cell objective's gradient (gpl_place_cells' search direction) against central
  differences of gpl_cell_objective, and the placement raising every cell's objective.
"""
import numpy as np
import pytest

from gaspacho2_b200 import GPLVM, synth
from gaspacho2_b200.encoder import Encoder, cell_objective, place_cells, procrustes_rmse, select_genes
from oracle import encoder_oracle as eo

pytestmark = pytest.mark.gpu


def _features(y, ls, genes, order):
    """Dense log1p(y / s) rows of the selected genes in the given cell order (the oracle's input)."""
    F = np.zeros((y.N, len(genes)))
    col = {int(g): f for f, g in enumerate(genes)}
    for g in genes:
        b, e = int(y.p[g]), int(y.p[g + 1])
        F[y.i[b:e], col[int(g)]] = np.log1p(y.x[b:e] / ls[y.i[b:e]])
    return F[order]


@pytest.fixture(scope="module")
def small():
    ds = synth.make(1, 5, N=2048, G=400, M=16, Q=5)
    genes = select_genes(ds.y, ds.ls, 200)
    order = np.random.default_rng(0).permutation(ds.N).astype(np.int32)
    return ds, genes, order


def test_encoder_gradients_match_oracle(small):
    ds, genes, order = small
    B = 512
    with Encoder(len(genes), ds.Q, hidden=256, batch=B, seed=3) as enc:
        enc.set_cells(0, ds.y, ds.ls, genes, order)
        enc.set_targets(ds.X_true)
        params = enc.get_params()
        for bi in (0, 2):
            loss, g = enc.grads(bi)
            rows = order[bi * B:(bi + 1) * B]
            F = _features(ds.y, ds.ls, genes, order)[bi * B:(bi + 1) * B]
            lo, go, _ = eo.loss_and_grads(params, F, ds.X_true[rows])
            assert abs(loss - lo) <= 1e-5 * abs(lo), (loss, lo)
            for k in go:
                e = np.linalg.norm(g[k] - go[k]) / max(np.linalg.norm(go[k]), 1e-30)
                print(f"batch {bi} {k}: rel L2 {e:.2e}")
                assert e <= 2e-3, (k, e)


def test_encoder_trains_and_predicts_unseen_cells(small):
    ds, genes, order = small
    train = order[:1536]
    test = order[1536:]
    with Encoder(len(genes), ds.Q, hidden=256, batch=512, seed=4) as enc:
        enc.set_cells(0, ds.y, ds.ls, genes, np.concatenate([train, test]).astype(np.int32))
        enc.set_targets(ds.X_true)
        losses = enc.train(40, lr=2e-3, seed=1)
        assert np.all(np.isfinite(losses))
        assert losses[-1] < losses[0] - 1.0, losses
        mean, lv = enc.predict(0)
        assert np.all(np.isfinite(mean)) and np.all(np.isfinite(lv))
        # the last 512 rows were never a training batch (3 whole batches of 512 cover 1536 rows)
        r_unseen = procrustes_rmse(mean[test], ds.X_true[test])
        r_null = procrustes_rmse(np.random.default_rng(0).standard_normal((len(test), ds.Q)), ds.X_true[test])
        print(f"unseen cells: Procrustes RMSE {r_unseen:.3f} (random {r_null:.3f})")
        assert r_unseen < 0.8 * r_null


@pytest.fixture(scope="module")
def fitted():
    ds = synth.make(0, 9, N=1200, G=120, M=12, Q=2)
    with GPLVM.from_dataset(ds) as m:
        m.set_params(ds.init)
        m.kernel_mats()
        m.glm_init()
        m.fit(1, 15)
        prm = {k: m.get(k) for k in ("Omega", "delta", "X", "T", "rho", "phi", "Beta")}
    return ds, prm


def _placement_ctx(ds, prm):
    m = GPLVM.from_dataset(ds)
    Q, M = ds.Q, ds.M
    from gaspacho2_b200.formats import Params

    m.set_params(Params(prm["Omega"], prm["delta"], prm["X"].reshape(Q, ds.N).T, prm["T"].reshape(Q, M).T,
                        prm["rho"], prm["phi"]))
    m.set_beta(prm["Beta"].reshape(-1, ds.J, order="F") if prm["Beta"].ndim == 1 else prm["Beta"])
    return m


def test_cell_objective_gradient_matches_differences(fitted):
    """The per-cell gradient (the direction the placement's L-BFGS follows) against central
    differences of the per-cell objective, every latent dimension of a few cells."""
    ds, prm = fitted
    with _placement_ctx(ds, prm) as m:
        X = prm["X"].reshape(ds.Q, ds.N).T.copy()
        f0, g = cell_objective(m, X, grad=True)
        assert np.all(np.isfinite(f0)) and np.all(np.isfinite(g))
        cells = np.random.default_rng(2).choice(ds.N, 8, replace=False)
        h = 1e-5
        for q in range(ds.Q):
            Xp, Xm = X.copy(), X.copy()
            Xp[cells, q] += h
            Xm[cells, q] -= h
            fd = (cell_objective(m, Xp)[cells] - cell_objective(m, Xm)[cells]) / (2 * h)
            err = np.abs(fd - g[cells, q]) / np.maximum(np.abs(fd), 1.0)
            print(f"dim {q}: max rel err {err.max():.2e}")
            assert np.all(err <= 1e-5), (q, fd, g[cells, q])


def test_placement_raises_objective_and_recovers_fitted_coordinates(fitted):
    ds, prm = fitted
    with _placement_ctx(ds, prm) as m:
        Xfit = prm["X"].reshape(ds.Q, ds.N).T.copy()
        f_fit = cell_objective(m, Xfit)
        start = Xfit + 0.5 * np.random.default_rng(3).standard_normal(Xfit.shape)
        f_start = cell_objective(m, start)
        Xp, f_end, st = place_cells(m, start, iters=30)
        assert st["steps"] == 30
        assert np.all(f_end >= f_start - 1e-9 * np.abs(f_start))
        gap_start = np.median((f_fit - f_start) / np.abs(f_fit))
        gap_end = np.median((f_fit - f_end) / np.abs(f_fit))
        print(f"median objective gap to the fitted X: start {gap_start:.2e}, after 30 steps {gap_end:.2e}")
        assert gap_end < 0.2 * gap_start


def test_amortised_placement_experiment_runs_end_to_end():
    """The whole experiment at configuration 0 (2,000 cells): fit, validation-chosen epochs,
    clamped predictions, placement from the encoder and from zero; every reported figure finite."""
    from gaspacho2_b200.encoder import amortised_placement

    out = amortised_placement(0, 1536, 464, 20, 40, n_genes=200, batch=256)
    for k in ("elbo_gap_encoder", "elbo_gap_without_encoder", "validation_rmse", "epochs_chosen",
              "clamped_fraction", "procrustes_rmse"):
        assert k in out, k
    assert 0 < out["epochs_chosen"] <= 40
    assert all(np.isfinite(r) for _, r in out["validation_rmse"])
    print({k: out[k] for k in ("elbo_gap_encoder", "elbo_gap_without_encoder", "cells_refined_above_start_from_zero",
                               "epochs_chosen", "clamped_fraction")})
    assert out["non_finite_cells"] <= 464 // 20, "non-finite objectives at more than 5% of the held-out cells"
    for k in ("elbo_gap_encoder", "elbo_gap_without_encoder"):
        assert np.isfinite(out[k]["median"]), k
    assert 0.0 <= out["clamped_fraction"] <= 1.0

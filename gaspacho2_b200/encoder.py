"""The amortised encoder over the C ABI (gpl_enc_*, include/gpl.h) and the per-cell placement
that judges it (gpl_place_cells).

The reference places every cell by L-BFGS on its latent coordinates (ggplvm.cu:1214-1301). The
encoder is trained on (cell profile, fitted X) pairs of a plain fit and predicts a new cell's
coordinates directly; the per-cell L-BFGS at the fitted model then refines that prediction
(fallback) and scores it (judge). Everything runs in the library's CUDA kernels; this module only
selects the feature genes, moves host arrays and drives the calls.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from ._lib import GplError

_dp = ctypes.POINTER(ctypes.c_double)
_fp = ctypes.POINTER(ctypes.c_float)
_ip = ctypes.POINTER(ctypes.c_int32)


def _d(a):
    return None if a is None else a.ctypes.data_as(_dp)


def select_genes(y, ls, n: int) -> np.ndarray:
    """The n genes with the largest variance of log1p(y / s) over cells (ties by gene index),
    from gene-major CSR counts; returned in increasing gene order."""
    N, J = int(y.N), int(y.J)
    s1 = np.zeros(J)
    s2 = np.zeros(J)
    p = np.asarray(y.p, np.int64)
    v = np.log1p(np.asarray(y.x, np.float64) / np.asarray(ls, np.float64)[np.asarray(y.i, np.int64)])
    gene = np.repeat(np.arange(J), np.diff(p))
    np.add.at(s1, gene, v)
    np.add.at(s2, gene, v * v)
    var = s2 / N - (s1 / N) ** 2
    top = np.argsort(-var, kind="stable")[:n]
    return np.sort(top).astype(np.int32)


class Encoder:
    """MLP n_in -> hidden -> hidden -> 2Q (mean, log-variance) on one CUDA device."""

    def __init__(self, n_in: int, Q: int, hidden: int = 256, batch: int = 1024, device: int = 0,
                 stream: Optional[int] = None, seed: int = 0):
        L = _lib.load()
        h = ctypes.c_void_p()
        rc = L.gpl_enc_create(ctypes.byref(h), int(device), ctypes.c_void_p(stream) if stream else None, int(n_in),
                              int(hidden), int(Q), int(batch), ctypes.c_uint64(seed))
        if rc != 0:
            raise GplError(f"gpl_enc_create: {_lib.ERRORS.get(rc, rc)}")
        self.h, self._L = h, L
        self.n_in, self.Q, self.hidden, self.batch = int(n_in), int(Q), int(hidden), int(batch)
        self.N = [0, 0]

    def close(self):
        if getattr(self, "h", None):
            self._L.gpl_enc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def _c(self, rc, what):
        if rc != 0:
            msg = self._L.gpl_enc_last_error(self.h)
            raise GplError(f"{what}: {_lib.ERRORS.get(rc, rc)} {msg.decode() if msg else ''}".strip())

    def set_cells(self, which: int, y, ls, genes, order=None):
        ci = np.ascontiguousarray(y.i, np.int32)
        gp = np.ascontiguousarray(y.p, np.int32)
        cx = np.ascontiguousarray(y.x, np.float64)
        g = np.ascontiguousarray(genes, np.int32)
        o = None if order is None else np.ascontiguousarray(order, np.int32)
        self._c(self._L.gpl_enc_set_cells(self.h, int(which), int(y.N), int(y.J), int(ci.shape[0]),
                                          ci.ctypes.data_as(_ip), gp.ctypes.data_as(_ip), _d(cx),
                                          _d(np.ascontiguousarray(ls, np.float64)), g.ctypes.data_as(_ip),
                                          None if o is None else o.ctypes.data_as(_ip)), "gpl_enc_set_cells")
        self.N[which] = int(y.N)

    def set_targets(self, X: np.ndarray):
        x = np.ascontiguousarray(np.asarray(X, np.float64).ravel(order="F"))
        self._c(self._L.gpl_enc_set_targets(self.h, _d(x)), "gpl_enc_set_targets")

    def n_params(self) -> int:
        n = ctypes.c_int64()
        self._c(self._L.gpl_enc_n_params(self.h, ctypes.byref(n)), "gpl_enc_n_params")
        return n.value

    def _unflat(self, a: np.ndarray) -> dict:
        H, n_in, Q2 = self.hidden, self.n_in, 2 * self.Q
        out, o = {}, 0
        for k, shape in (("W1", (H, n_in)), ("b1", (H,)), ("W2", (H, H)), ("b2", (H,)), ("W3", (Q2, H)),
                         ("b3", (Q2,))):
            n = int(np.prod(shape))
            out[k] = a[o:o + n].reshape(shape).astype(np.float64)
            o += n
        return out

    def get_params(self) -> dict:
        a = np.zeros(self.n_params(), np.float32)
        self._c(self._L.gpl_enc_get_params(self.h, a.ctypes.data_as(_fp)), "gpl_enc_get_params")
        return self._unflat(a)

    def set_params(self, params: dict):
        a = np.concatenate([np.asarray(params[k], np.float32).ravel() for k in ("W1", "b1", "W2", "b2", "W3", "b3")])
        self._c(self._L.gpl_enc_set_params(self.h, a.ctypes.data_as(_fp)), "gpl_enc_set_params")

    def grads(self, batch_index: int = 0):
        """(mean loss, gradients) of one training batch, parameters unchanged."""
        loss = ctypes.c_double()
        a = np.zeros(self.n_params(), np.float32)
        self._c(self._L.gpl_enc_grads(self.h, int(batch_index), ctypes.byref(loss), a.ctypes.data_as(_fp)),
                "gpl_enc_grads")
        return loss.value, self._unflat(a)

    def train(self, epochs: int, lr: float = 1e-3, seed: int = 0) -> np.ndarray:
        losses = np.zeros(max(1, epochs))
        self._c(self._L.gpl_enc_train(self.h, int(epochs), float(lr), ctypes.c_uint64(seed), _d(losses)),
                "gpl_enc_train")
        return losses[:epochs]

    def predict(self, which: int = 1):
        N, Q = self.N[which], self.Q
        mean = np.zeros(N * Q)
        lv = np.zeros(N * Q)
        self._c(self._L.gpl_enc_predict(self.h, int(which), _d(mean), _d(lv)), "gpl_enc_predict")
        return mean.reshape(Q, N).T.copy(), lv.reshape(Q, N).T.copy()

    def launches(self) -> int:
        n = ctypes.c_int64()
        self._c(self._L.gpl_enc_launch_count(self.h, ctypes.byref(n)), "gpl_enc_launch_count")
        return n.value


def place_cells(model, X0: np.ndarray, iters: int = 30):
    """Per-cell L-BFGS placement (gpl_place_cells) on a GPLVM context that holds the new cells and
    the fitted T, rho, delta and beta. Returns (X, per-cell objective, stats)."""
    X = np.ascontiguousarray(np.asarray(X0, np.float64).ravel(order="F"))
    obj = np.zeros(model.N)
    st = (ctypes.c_int32 * 3)()
    model._c(model._L.gpl_place_cells(model.h, int(iters), _d(X), _d(obj), st), "gpl_place_cells")
    return X.reshape(model.Q, model.N).T.copy(), obj, {"steps": st[0], "evals": st[1], "tries": st[2]}


def cell_objective(model, X: np.ndarray, grad: bool = False):
    """Per-cell objective at X (N x Q); with grad, also its gradient (N x Q)."""
    x = np.ascontiguousarray(np.asarray(X, np.float64).ravel(order="F"))
    obj = np.zeros(model.N)
    g = np.zeros(model.N * model.Q) if grad else None
    model._c(model._L.gpl_cell_objective(model.h, _d(x), _d(obj), _d(g)), "gpl_cell_objective")
    return (obj, g.reshape(model.Q, model.N).T.copy()) if grad else obj


def amortised_placement(config: int, n_train: int, n_test: int, fit_lbfgs: int, epochs: int, n_genes: int = 2000,
                        hidden: int = 256, batch: int = 1024, iters: int = 30, seed: int = 0, device: int = 0,
                        stream: Optional[int] = None, precision: str = "fp64", lr: float = 1e-3, G=None):
    """The encoder's experiment: a plain fit on n_train cells of configuration `config`, the
    encoder trained on (profile, fitted X) of nine tenths of those cells for up to `epochs`
    epochs, keeping the parameters of the 20-epoch checkpoint with the smallest RMSE on the
    other tenth; then n_test held-out cells of the same generator and gene parameters placed
    (a) by the encoder alone (clamped to the training targets' box), (b) by the encoder followed
    by `iters` per-cell L-BFGS steps at the fitted model (the fallback, whose result is the
    judge), (c) by the same steps from X = 0 (the method without the encoder). Returns a dict of
    the per-cell objective gaps (relative to the judge), Procrustes-aligned RMSEs and timings."""
    import time

    from . import synth
    from .formats import Params
    from .model import GPLVM

    kw = {"N": n_train + n_test}
    if G:
        kw["G"] = G
    full = synth.make(config, seed, init=False, **kw)
    train = synth.cell_subset(full, np.arange(n_train))
    test = synth.cell_subset(full, np.arange(n_train, n_train + n_test), init=False)
    out = {"config": config, "n_train": n_train, "n_test": n_test, "G": full.J, "M": full.M, "Q": full.Q,
           "fit_lbfgs": fit_lbfgs, "epochs": epochs, "n_genes": n_genes, "hidden": hidden, "batch": batch,
           "refine_iters": iters, "precision": precision}
    t0 = time.time()
    with GPLVM.from_dataset(train, device=device, stream=stream, precision=precision) as m:
        m.set_params(train.init)
        m.kernel_mats()
        m.glm_init()
        rc, st, tr = m.fit(100000, fit_lbfgs)
        fit = {k: m.get(k) for k in ("delta", "X", "T", "rho", "phi", "Beta")}
        out["fit_seconds"] = time.time() - t0
        out["fit_final_objective"] = float(tr[-1]) if len(tr) else None
        # the plain method's per-cell coordinates of the training cells: the fit's X refined by
        # the per-cell L-BFGS at the fitted model (the judge's own criterion), the encoder's targets
        Q, M, N1, N2 = full.Q, full.M, n_train, n_test
        t0 = time.time()
        Xfit, l_train, _ = place_cells(m, fit["X"].reshape(Q, N1).T.copy(), iters)
        out["target_refine_seconds"] = time.time() - t0
    genes = select_genes(train.y, train.ls, min(n_genes, full.J))
    # a tenth of the training cells (at least one batch) held out to choose the epoch count
    n_val = max(batch, n_train // 10)
    rng = np.random.default_rng(seed + 1)
    split = rng.permutation(N1)
    tr_idx, va_idx = np.sort(split[n_val:]), np.sort(split[:n_val])
    fit_cells = synth.cell_subset(train, tr_idx, init=False)
    val_cells = synth.cell_subset(train, va_idx, init=False)
    perm = rng.permutation(tr_idx.shape[0]).astype(np.int32)
    t0 = time.time()
    chunk = max(1, min(epochs, 20))
    with Encoder(len(genes), Q, hidden=hidden, batch=batch, device=device, stream=stream, seed=seed) as enc:
        enc.set_cells(0, fit_cells.y, fit_cells.ls, genes, perm)
        enc.set_targets(Xfit[tr_idx])
        enc.set_cells(1, val_cells.y, val_cells.ls, genes)
        losses, val_rmse, best, best_params, best_epochs, done = [], [], np.inf, None, 0, 0
        while done < epochs:
            k = min(chunk, epochs - done)
            losses.extend(enc.train(k, lr=lr, seed=seed + done).tolist())
            done += k
            mv, _ = enc.predict(1)
            r = float(np.sqrt(np.mean((mv - Xfit[va_idx]) ** 2)))
            val_rmse.append([done, r])
            if r < best:
                best, best_params, best_epochs = r, enc.get_params(), done
        if best_params is not None:
            enc.set_params(best_params)
        out["train_seconds"] = time.time() - t0
        out["train_loss_first_last"] = [float(losses[0]), float(losses[-1])] if len(losses) else None
        out["validation_rmse"] = val_rmse
        out["epochs_chosen"] = best_epochs
        enc.set_cells(1, test.y, test.ls, genes)
        t0 = time.time()
        X_enc, _ = enc.predict(1)
        out["encoder_seconds"] = time.time() - t0
        out["encoder_launches"] = enc.launches()
    # predictions outside the training targets' box (widened by a tenth of its width per
    # dimension) are clamped to it: the encoder has seen no cell there
    lo, hi = Xfit.min(0), Xfit.max(0)
    lo, hi = lo - 0.1 * (hi - lo), hi + 0.1 * (hi - lo)
    out["clamped_fraction"] = float(np.mean(np.any((X_enc < lo) | (X_enc > hi), axis=1)))
    X_enc = np.clip(X_enc, lo, hi)
    prm = Params(np.ones(N2), fit["delta"], X_enc, fit["T"].reshape(Q, M).T, fit["rho"], fit["phi"])
    with GPLVM.from_dataset(test, device=device, stream=stream) as jm:
        jm.set_params(prm)
        jm.set_beta(fit["Beta"].reshape(full.J, -1).T)
        l_enc = cell_objective(jm, X_enc)
        t0 = time.time()
        X_ref, l_ref, st_ref = place_cells(jm, X_enc, iters)
        out["refine_seconds"] = time.time() - t0
        X_zero, l_zero, st_zero = place_cells(jm, np.zeros_like(X_enc), iters)
        l_true = cell_objective(jm, test.X_true)
    # gaps over the cells whose objectives are finite at every point compared (the count of the
    # others is reported)
    ok = np.isfinite(l_ref) & np.isfinite(l_enc) & np.isfinite(l_zero)
    out["non_finite_cells"] = int(np.sum(~ok))
    rel = lambda a: (l_ref[ok] - a[ok]) / np.abs(l_ref[ok])  # noqa: E731
    g_enc, g_zero = rel(l_enc), rel(l_zero)
    stat = lambda g: {"median": float(np.median(g)), "mean": float(np.mean(g)),  # noqa: E731
                      "p95": float(np.quantile(g, 0.95))} if g.size else {"median": None, "mean": None, "p95": None}
    out["elbo_gap_encoder"] = stat(g_enc)
    out["elbo_gap_without_encoder"] = {**stat(g_zero), "note": f"{iters} per-cell L-BFGS steps from X = 0"}
    out["cells_refined_above_start_from_zero"] = float(np.mean(l_ref[ok] > l_zero[ok])) if ok.any() else None
    out["procrustes_rmse"] = {"encoder_vs_judge": procrustes_rmse(X_enc, X_ref),
                              "encoder_vs_truth": procrustes_rmse(X_enc, test.X_true),
                              "judge_vs_truth": procrustes_rmse(X_ref, test.X_true),
                              "without_encoder_vs_truth": procrustes_rmse(X_zero, test.X_true)}
    ok_t = ok & np.isfinite(l_true)
    out["objective_at_true_X_gap_median"] = (float(np.median((l_ref[ok_t] - l_true[ok_t]) / np.abs(l_ref[ok_t])))
                                             if ok_t.any() else None)
    out["placement_stats"] = {"refine": st_ref, "from_zero": st_zero}
    return out


def procrustes_rmse(A: np.ndarray, B: np.ndarray) -> float:
    """RMSE between A and B after the orthogonal rotation, scaling and shift of A that best
    matches B (both N x Q)."""
    a = A - A.mean(0)
    b = B - B.mean(0)
    U, s, Vt = np.linalg.svd(a.T @ b)
    R = U @ Vt
    scale = s.sum() / max((a * a).sum(), 1e-300)
    return float(np.sqrt(np.mean((scale * a @ R - b) ** 2)))

"""Host-side mirror of the reference driver's phases over the C ABI (include/gpl.h).

``GPLVM`` keeps the reference's vocabulary: the phases are the reference kernels' names
(kernel matrices, GLM init, IRLS sweep, objective, gradient, L-BFGS update, downdate) and
``get(name)`` returns the reference's buffers in the reference's layouts, so a test can
run the same sequence through this class, the reference build (oracle/_ref) and the
oracle and compare buffer by buffer.
"""
from __future__ import annotations

import ctypes
from typing import Optional

import numpy as np

from . import _lib
from ._lib import check

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int32)


def _d(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_dp)


class GPLVM:
    """One fit context on a CUDA device: counts, design and the state of the fit."""

    def __init__(self, y, z, ls, X0, M: int, Q: int, device: int = 0, stream: Optional[int] = None,
                 precision: str = "fp64"):
        L = _lib.load()
        h = ctypes.c_void_p()
        check(L.gpl_create(ctypes.byref(h), int(device), ctypes.c_void_p(stream) if stream else None), None,
              "gpl_create")
        self.h = h
        self._L = L
        ci = np.ascontiguousarray(y.i, np.int32)
        gp = np.ascontiguousarray(y.p, np.int32)
        cx = np.ascontiguousarray(y.x, np.float64)
        check(L.gpl_load_counts(h, int(y.N), int(y.J), int(ci.shape[0]), ci.ctypes.data_as(_ip),
                                gp.ctypes.data_as(_ip), _d(cx)), h, "gpl_load_counts")
        c = np.ascontiguousarray(z.c, np.int32)
        v = np.ascontiguousarray(z.v, np.int32)
        body = z.body_bytes()
        buf = ctypes.create_string_buffer(body, max(1, len(body)))
        check(L.gpl_load_design(h, int(z.N), int(z.n_var), c.ctypes.data_as(_ip), v.ctypes.data_as(_ip),
                                ctypes.cast(buf, ctypes.c_void_p), len(body), int(M), int(Q)), h, "gpl_load_design")
        check(L.gpl_set_size_factors(h, _d(np.ascontiguousarray(ls, np.float64))), h, "gpl_set_size_factors")
        X = np.ascontiguousarray(np.asarray(X0, np.float64).ravel(order="F"))
        check(L.gpl_set_params(h, None, None, _d(X), None, None, None), h, "gpl_set_params")
        d = (ctypes.c_int32 * 6)()
        check(L.gpl_dims(h, d), h, "gpl_dims")
        self.N, self.J, self.M, self.P, self.p, self.Q = list(d)
        self.set_precision(precision)

    @classmethod
    def from_dataset(cls, ds, **kw) -> "GPLVM":
        return cls(ds.y, ds.z, ds.ls, ds.X0, ds.M, ds.Q, **kw)

    # -- lifetime ------------------------------------------------------------------------------
    def close(self):
        if getattr(self, "h", None):
            self._L.gpl_destroy(self.h)
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
        check(rc, self.h, what)

    # -- parameters ----------------------------------------------------------------------------
    def set_precision(self, precision: str):
        self._c(self._L.gpl_set_precision(self.h, _lib.PREC[precision]), "gpl_set_precision")

    def set_option(self, name: str, value: int) -> None:
        """A named integer option of the context (gpl_set_option)."""
        self._c(self._L.gpl_set_option(self.h, name.encode(), int(value)), f"gpl_set_option({name})")

    def get_option(self, name: str) -> int:
        v = ctypes.c_int64()
        self._c(self._L.gpl_get_option(self.h, name.encode(), ctypes.byref(v)), f"gpl_get_option({name})")
        return v.value

    def tuning(self, name: str) -> dict:
        """The autotuner's record of one choice: the chosen value (None while open) and each
        candidate's best measured launch time in ms (None if untimed)."""
        chosen = ctypes.c_int32()
        n = ctypes.c_int32()
        cands = (ctypes.c_int32 * 16)()
        ms = (ctypes.c_double * 16)()
        self._c(self._L.gpl_tuning(self.h, name.encode(), ctypes.byref(chosen), cands, ms, 16, ctypes.byref(n)),
                f"gpl_tuning({name})")
        return {"chosen": None if chosen.value < 0 else chosen.value,
                "candidates_ms": {int(cands[k]): (ms[k] if ms[k] >= 0 else None) for k in range(n.value)}}

    def set_params(self, prm) -> None:
        flat = [np.ascontiguousarray(a, dtype=np.float64) for a in prm.flat()]
        self._keep = flat
        self._c(self._L.gpl_set_params(self.h, *[_d(a) for a in flat]), "gpl_set_params")

    def set_beta(self, beta: np.ndarray) -> None:
        b = np.ascontiguousarray(np.asarray(beta, np.float64).ravel(order="F"))
        self._c(self._L.gpl_set_beta(self.h, _d(b)), "gpl_set_beta")

    def n_params(self) -> int:
        return self.N + self.p + self.N * self.Q + self.M * self.Q + self.Q

    # -- phases (reference driver order, ggplvm.cu:1101-1330) -------------------------------------
    def kernel_mats(self):
        self._c(self._L.gpl_kernel_mats(self.h), "gpl_kernel_mats")

    def glm_init(self):
        self._c(self._L.gpl_glm_init(self.h), "gpl_glm_init")

    def gram(self):
        """getPsi alone: every gene's Gram at the current W, Omega and DeltaInv (no factorization)."""
        self._c(self._L.gpl_gram(self.h), "gpl_gram")

    def expand_delta(self):
        self._c(self._L.gpl_expand_delta(self.h), "gpl_expand_delta")

    def irls_sweep(self, itr: int, jtr: int) -> float:
        v = ctypes.c_double()
        self._c(self._L.gpl_irls_sweep(self.h, int(jtr), ctypes.byref(v)), "gpl_irls_sweep")
        return v.value

    def irls(self, itr: int, jtr_max: int) -> int:
        n = ctypes.c_int()
        rc = self._L.gpl_irls(self.h, int(jtr_max), ctypes.byref(n))
        if rc == -5:
            return -1
        self._c(rc, "gpl_irls")
        return n.value

    def objective_after_irls(self, itr: int = 0) -> float:
        v = ctypes.c_double()
        self._c(self._L.gpl_objective_after_irls(self.h, ctypes.byref(v)), "gpl_objective_after_irls")
        return v.value

    def objective(self, itr: int, slot: int) -> float:
        v = ctypes.c_double()
        self._c(self._L.gpl_objective(self.h, int(slot), ctypes.byref(v)), "gpl_objective")
        return v.value

    def gradient(self) -> np.ndarray:
        g = np.zeros(self.n_params())
        self._c(self._L.gpl_gradient(self.h, _d(g)), "gpl_gradient")
        return g

    def lbfgs_update(self, jtr: int, rhoflag: int):
        self._c(self._L.gpl_lbfgs_update(self.h, int(jtr), int(rhoflag)), "gpl_lbfgs_update")

    def downdate(self, jtr: int, sr: float, rhoflag: int):
        self._c(self._L.gpl_downdate(self.h, int(jtr), float(sr), int(rhoflag)), "gpl_downdate")

    def beta_from_tilde(self):
        self._c(self._L.gpl_beta_from_tilde(self.h), "gpl_beta_from_tilde")

    def fit(self, itr_max: int, lbfgs_budget: int, trace_cap: int = 100000):
        st = (ctypes.c_int32 * 4)()
        tr = np.zeros(trace_cap)
        rc = self._L.gpl_fit(self.h, int(itr_max), int(lbfgs_budget), st, _d(tr), int(trace_cap))
        if rc not in (0, -5):
            self._c(rc, "gpl_fit")
        stats = dict(outer=st[0], irls=st[1], lbfgs=st[2], evals=st[3])
        return (1 if rc == -5 else 0), stats, tr[:stats["outer"] + stats["lbfgs"]].copy()

    def fit_outer(self, itr: int, lbfgs_budget: int = 0, trace_cap: int = 20000):
        """One outer iteration of the driver (gpl_fit_outer): (rc, stats, trace) with stats
        {irls, lbfgs, evals} of this iteration and its accepted objective values."""
        st = (ctypes.c_int32 * 4)()
        tr = np.zeros(trace_cap)
        rc = self._L.gpl_fit_outer(self.h, int(itr), int(lbfgs_budget), st, _d(tr), int(trace_cap))
        if rc not in (0, -5):
            self._c(rc, "gpl_fit_outer")
        return (1 if rc == -5 else 0), dict(irls=st[0], lbfgs=st[1], evals=st[2]), tr[:st[3]].copy()

    # -- the differential-expression driver's model comparison (ggplvm_de.cu) ------------------
    def de_model(self, model) -> None:
        """Select the DE driver's model: "null" (no GP), "full" (the GP over every latent
        dimension) or a latent dimension q (the GP over dimension q alone)."""
        code = {"null": _lib.DE_NULL, "full": _lib.DE_FULL}.get(model, model)
        self._c(self._L.gpl_de_model(self.h, int(code)), "gpl_de_model")

    def de_irls(self, jtr_max: int = 1000, tol: float = 1e-8, trace_cap: int = 0):
        """The selected model's GLM initialisation and IRLS in the DE driver's forms; returns
        (per-gene log-likelihoods, sweeps, summed likelihood per sweep)."""
        lk = np.zeros(self.J)
        n = ctypes.c_int32()
        tr = np.zeros(max(1, trace_cap))
        self._c(self._L.gpl_de_irls(self.h, int(jtr_max), float(tol), _d(lk), ctypes.byref(n),
                                    _d(tr) if trace_cap else None, int(trace_cap)), "gpl_de_irls")
        return lk, n.value, tr[:min(n.value, trace_cap)].copy()

    def vc_fit(self, itr_max: int = 100, lbfgs_max: int = 100):
        """The variance-component driver (ggplvm_delta.cu) from the parameters set: refits
        delta[p-2]; returns (delta[p-2], objective) after each outer iteration."""
        dg = np.zeros(itr_max)
        obj = np.zeros(itr_max)
        n = ctypes.c_int32()
        self._c(self._L.gpl_vc_fit(self.h, int(itr_max), int(lbfgs_max), _d(dg), _d(obj), int(itr_max),
                                   ctypes.byref(n)), "gpl_vc_fit")
        return dg[:n.value].copy(), obj[:n.value].copy()

    def evaluate(self, params: np.ndarray, grad_out: Optional[np.ndarray] = None):
        """Objective and gradient at natural-scale params [Omega | delta | X | T | rho]."""
        params = np.ascontiguousarray(params, np.float64)
        g = grad_out if grad_out is not None else np.zeros(self.n_params())
        v = ctypes.c_double()
        self._c(self._L.gpl_evaluate(self.h, _d(params), int(params.shape[0]), ctypes.byref(v), _d(g)),
                "gpl_evaluate")
        return v.value, g

    def init_latent(self, pca_iters: int = 60, kmeans_iters: int = 25, seed: int = 0):
        """The start from the counts (gpl_init_latent): X (N x Q) PCA scores of log1p(y / s) at unit
        variance, T (M x Q) k-means centres of X."""
        X = np.zeros(self.N * self.Q)
        T = np.zeros(self.M * self.Q)
        self._c(self._L.gpl_init_latent(self.h, int(pca_iters), int(kmeans_iters), ctypes.c_uint64(seed), _d(X),
                                        _d(T)), "gpl_init_latent")
        return X.reshape(self.Q, self.N).T.copy(), T.reshape(self.Q, self.M).T.copy()

    def cis_stats(self, dosages: np.ndarray, donor_var: int):
        """Per-(gene, variant) statistics (gpl_cis_stats) for donor dosages [donors][genes][variants]:
        returns (S, LR), both J x V."""
        dos = np.ascontiguousarray(dosages, np.int8)
        D, J, V = dos.shape
        S = np.zeros(J * V)
        LR = np.zeros(J * V)
        self._c(self._L.gpl_cis_stats(self.h, int(donor_var), int(D), int(V), dos.ctypes.data_as(ctypes.c_void_p),
                                      _d(S), _d(LR)), "gpl_cis_stats")
        return S.reshape(V, J).T.copy(), LR.reshape(V, J).T.copy()

    def score_stats(self, G: np.ndarray) -> np.ndarray:
        """Genotype score statistics (getScoreStats, ggplvm_de.cu:489-535): G is N x L, the
        result J x L, at the current fitted state."""
        G = np.asfortranarray(G, dtype=np.float64)
        L = G.shape[1]
        S = np.zeros(self.J * L)
        self._c(self._L.gpl_score_stats(self.h, int(L), _d(np.ascontiguousarray(G.ravel(order="F"))), _d(S)),
                "gpl_score_stats")
        return S.reshape(L, self.J).T

    def evaluate_device(self):
        """Enqueues one objective+gradient evaluation at the device-resident parameters."""
        self._c(self._L.gpl_evaluate_device(self.h), "gpl_evaluate_device")

    # -- state ---------------------------------------------------------------------------------
    def get(self, name: str) -> np.ndarray:
        n = ctypes.c_int64()
        self._c(self._L.gpl_get(self.h, name.encode(), None, 0, ctypes.byref(n)), f"gpl_get({name})")
        out = np.zeros(n.value)
        self._c(self._L.gpl_get(self.h, name.encode(), _d(out), n.value, ctypes.byref(n)), f"gpl_get({name})")
        return out

    def n_dense(self) -> int:
        """Number of dense model columns (intercept, numerics, one-hots kept dense, Knm)."""
        n = ctypes.c_int64()
        self._c(self._L.gpl_get(self.h, b"Dm", None, 0, ctypes.byref(n)), "gpl_get(Dm)")
        return n.value // self.N

    def params_vector(self) -> np.ndarray:
        return np.concatenate([self.get(k) for k in ("Omega", "delta", "X", "T", "rho")])

    def profile(self, on: bool = True):
        self._c(self._L.gpl_profile_enable(self.h, int(on)), "gpl_profile_enable")

    def profile_reset(self):
        self._c(self._L.gpl_profile_reset(self.h), "gpl_profile_reset")

    def profile_read(self, name: str):
        ms = ctypes.c_double()
        n = ctypes.c_int64()
        self._c(self._L.gpl_profile_read(self.h, name.encode(), ctypes.byref(ms), ctypes.byref(n)),
                "gpl_profile_read")
        return ms.value, n.value

    def launches(self) -> int:
        n = ctypes.c_int64()
        self._c(self._L.gpl_launch_count(self.h, ctypes.byref(n)), "gpl_launch_count")
        return n.value

    def sync(self):
        self._c(self._L.gpl_sync(self.h), "gpl_sync")

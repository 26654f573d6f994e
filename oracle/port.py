"""TEST INFRASTRUCTURE ONLY: ctypes driver for the oracle's C restatement (gpl_oracle.c).

Same method set as ``oracle.refcpu.RefModel`` and the product's ``gaspacho2_b200.GPLVM`` so a
test can run one sequence of phases through all three. Only tests, ``smoke()`` and
bench.py's CPU legs may load this module.
"""
from __future__ import annotations

import ctypes
import os
from typing import Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ORACLE_SO = os.path.join(HERE, "_build", "libgpl_oracle.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)
_lib = None


def available() -> bool:
    return os.path.exists(ORACLE_SO)


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{ORACLE_SO} is not built (make -C oracle oracle)")
        L = ctypes.CDLL(ORACLE_SO)
        L.orc_create.restype = ctypes.c_void_p
        L.orc_create.argtypes = [ctypes.c_int, ctypes.c_int, ctypes.c_long, _ip, _ip, _dp, ctypes.c_int, _ip, _ip,
                                 ctypes.c_void_p, ctypes.c_long, ctypes.c_int, ctypes.c_int, _dp, _dp]
        L.orc_destroy.argtypes = [ctypes.c_void_p]
        L.orc_dims.argtypes = [ctypes.c_void_p, _ip]
        L.orc_init_params.argtypes = [ctypes.c_void_p]
        L.orc_set_params.argtypes = [ctypes.c_void_p] + [_dp] * 6
        L.orc_set_beta.argtypes = [ctypes.c_void_p, _dp]
        for name in ("orc_kernel_mats", "orc_glm_init", "orc_expand_delta", "orc_beta_from_tilde"):
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.orc_irls_sweep.restype = ctypes.c_double
        L.orc_irls_sweep.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_irls.restype = ctypes.c_int
        L.orc_irls.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_objective_after_irls.restype = ctypes.c_double
        L.orc_objective_after_irls.argtypes = [ctypes.c_void_p]
        L.orc_gradient.argtypes = [ctypes.c_void_p, _dp]
        L.orc_objective.restype = ctypes.c_double
        L.orc_objective.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_lbfgs_update.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.orc_downdate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.orc_fit.restype = ctypes.c_int
        L.orc_fit.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _ip, _dp, ctypes.c_int]
        L.orc_get.restype = ctypes.c_long
        L.orc_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _dp]
        L.orc_score_stats.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.orc_set_threads.argtypes = [ctypes.c_int]
        L.orc_kernel_mats_lv.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.orc_de_irls.restype = ctypes.c_int
        L.orc_de_irls.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double]
        L.orc_ta_equispaced.argtypes = [ctypes.c_int, ctypes.c_int, _dp]
        L.orc_vc_fit.restype = ctypes.c_int
        L.orc_vc_fit.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _dp, _dp, ctypes.c_int]
        _lib = L
    return _lib


def _dptr(a: Optional[np.ndarray]):
    return None if a is None else a.ctypes.data_as(_dp)


def set_threads(n: int) -> None:
    lib().orc_set_threads(int(n))


class OracleModel:
    def __init__(self, y, z, ls, X0, M: int, Q: int):
        L = lib()
        self._ci = np.ascontiguousarray(y.i, np.int32)
        self._gp = np.ascontiguousarray(y.p, np.int32)
        self._cx = np.ascontiguousarray(y.x, np.float64)
        self._c = np.ascontiguousarray(z.c, np.int32)
        self._v = np.ascontiguousarray(z.v, np.int32)
        body = z.body_bytes()
        self._body = ctypes.create_string_buffer(body, len(body) or 1)
        self._ls = np.ascontiguousarray(ls, np.float64)
        self._X0 = np.ascontiguousarray(np.asarray(X0, np.float64).ravel(order="F"))
        self.h = L.orc_create(y.N, y.J, y.L, self._ci.ctypes.data_as(_ip), self._gp.ctypes.data_as(_ip),
                              _dptr(self._cx), z.n_var, self._c.ctypes.data_as(_ip), self._v.ctypes.data_as(_ip),
                              ctypes.cast(self._body, ctypes.c_void_p), len(body), int(M), int(Q), _dptr(self._ls),
                              _dptr(self._X0))
        if not self.h:
            raise ValueError("oracle rejected the inputs")
        d = (ctypes.c_int * 6)()
        L.orc_dims(self.h, d)
        self.N, self.J, self.M, self.P, self.p, self.Q = list(d)

    @classmethod
    def from_dataset(cls, ds) -> "OracleModel":
        return cls(ds.y, ds.z, ds.ls, ds.X0, ds.M, ds.Q)

    def close(self):
        if self.h:
            lib().orc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_params(self, prm) -> None:
        flat = [np.ascontiguousarray(a, dtype=np.float64) for a in prm.flat()]
        lib().orc_set_params(self.h, *[_dptr(a) for a in flat])

    def set_beta(self, beta: np.ndarray) -> None:
        b = np.ascontiguousarray(np.asarray(beta, np.float64).ravel(order="F"))
        lib().orc_set_beta(self.h, _dptr(b))

    def kernel_mats(self):
        lib().orc_kernel_mats(self.h)

    def glm_init(self):
        lib().orc_glm_init(self.h)

    def expand_delta(self):
        lib().orc_expand_delta(self.h)

    def irls_sweep(self, itr: int, jtr: int) -> float:
        return lib().orc_irls_sweep(self.h, jtr)

    def irls(self, itr: int, jtr_max: int) -> int:
        return lib().orc_irls(self.h, jtr_max)

    def objective_after_irls(self, itr: int = 0) -> float:
        return lib().orc_objective_after_irls(self.h)

    def objective(self, itr: int, slot: int) -> float:
        return lib().orc_objective(self.h, slot)

    def gradient(self) -> np.ndarray:
        n = self.N + self.p + self.N * self.Q + self.M * self.Q + self.Q
        g = np.zeros(n)
        lib().orc_gradient(self.h, _dptr(g))
        return g

    def lbfgs_update(self, jtr: int, rhoflag: int):
        lib().orc_lbfgs_update(self.h, jtr, rhoflag)

    def downdate(self, jtr: int, sr: float, rhoflag: int):
        lib().orc_downdate(self.h, jtr, sr, rhoflag)

    def beta_from_tilde(self):
        lib().orc_beta_from_tilde(self.h)

    def fit(self, itr_max: int, lbfgs_budget: int, trace_cap: int = 100000):
        st = (ctypes.c_int * 4)()
        tr = np.zeros(trace_cap)
        rc = lib().orc_fit(self.h, itr_max, lbfgs_budget, st, _dptr(tr), trace_cap)
        stats = dict(outer=st[0], irls=st[1], lbfgs=st[2], evals=st[3])
        return rc, stats, tr[:stats["outer"] + stats["lbfgs"]].copy()

    def score_stats(self, G: np.ndarray) -> np.ndarray:
        """getScoreStats (ggplvm_de.cu:489-535): G is N x L, the result J x L."""
        G = np.asfortranarray(G, dtype=np.float64)
        L = G.shape[1]
        S = np.zeros(self.J * L)
        lib().orc_score_stats(self.h, L, _dptr(np.ascontiguousarray(G.ravel(order="F"))), _dptr(S))
        return S.reshape(L, self.J).T

    def get(self, name: str) -> np.ndarray:
        n = lib().orc_get(self.h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        lib().orc_get(self.h, name.encode(), _dptr(out))
        return out


def ta_equispaced(M: int, Q: int) -> np.ndarray:
    """initTaEquispaced (util.c:57-71): M x Q inducing points, column-major."""
    T = np.zeros(M * Q)
    lib().orc_ta_equispaced(int(M), int(Q), _dptr(T))
    return T.reshape(Q, M).T.copy()


def de_bfs(ds, prm, Mredc: int, Mfull: int, jtr_max: int = 1000):
    """The DE driver's model comparison (ggplvm_de.cu:1067-1207) on the oracle: per-gene
    log-likelihoods J x (Q + 2) of the null model, the Q one-dimension GP models (Mredc
    equispaced inducing points) and the full model (Mfull inducing points, prm.T), each
    refitted by the DE driver's IRLS at prm's Omega, delta, X and rho; phi starts at 1 and
    carries from model to model. Returns (BFs, sweeps per model, full-model beta P x J, phi)."""
    Q, J = ds.Q, ds.J
    BFs = np.zeros((J, Q + 2))
    sweeps = []
    phi = np.ones(J)
    delta = np.asarray(prm.delta, np.float64)

    def run(M, T, delta_m, lv, tol):
        nonlocal phi
        m = OracleModel(ds.y, ds.z, ds.ls, prm.X, M, Q)
        try:
            lib().orc_set_params(m.h, _dptr(np.ascontiguousarray(prm.Omega, np.float64)),
                                 _dptr(np.ascontiguousarray(delta_m)), _dptr(np.ascontiguousarray(
                                     np.asarray(prm.X, np.float64).ravel(order="F"))),
                                 _dptr(None if T is None else np.ascontiguousarray(np.asarray(T).ravel(order="F"))),
                                 _dptr(np.ascontiguousarray(prm.rho, np.float64)), _dptr(phi.copy()))
            if M > 0:
                lib().orc_kernel_mats_lv(m.h, int(lv))
            n = lib().orc_de_irls(m.h, int(jtr_max), float(tol))
            out = m.get("lkhds").copy()
            phi = m.get("phi").copy()
            beta = m.get("Beta").reshape(J, m.P).T.copy()
            return n, out, beta
        finally:
            m.close()

    n, BFs[:, 0], _ = run(0, None, delta[:-1].copy(), -1, 1e-5)
    sweeps.append(n)
    Tr = ta_equispaced(Mredc, Q)
    beta = None
    for q in range(Q):
        n, BFs[:, q + 1], _ = run(Mredc, Tr, delta, q, 1e-8)
        sweeps.append(n)
    n, BFs[:, Q + 1], beta = run(Mfull, np.asarray(prm.T), delta, -1, 1e-8)
    sweeps.append(n)
    return BFs, sweeps, beta, phi


def vc_fit(ds, prm, init_dg: float = 0.01, itr_max: int = 100, lbfgs_max: int = 100):
    """The variance-component driver (ggplvm_delta.cu:784-1097) on the oracle. ``ds`` holds the
    design with the extra variable last (its variance is refitted); ``prm`` the fit's Omega,
    X, T, rho and its p - 1 deltas (without the extra variable), as the driver reads them from
    params.bin. delta[p-2] starts at init_dg and delta[p-1] keeps initParams' value, as the
    driver leaves them. Returns (delta[p-2] after each outer iteration, the objective after
    each outer iteration)."""
    m = OracleModel(ds.y, ds.z, ds.ls, prm.X, ds.M, ds.Q)
    try:
        p = m.p
        d = m.get("delta")[:p].copy()  # initParams' values (init.cu:27-48)
        dfile = np.asarray(prm.delta, np.float64)
        d[:p - 2] = dfile[:p - 2]
        d[p - 2] = init_dg
        arr = [np.ascontiguousarray(np.asarray(a, np.float64).ravel(order="F")) for a in (prm.Omega, prm.X, prm.T, prm.rho)]
        lib().orc_set_params(m.h, _dptr(arr[0]), _dptr(np.ascontiguousarray(d)), _dptr(arr[1]), _dptr(arr[2]),
                             _dptr(arr[3]), None)
        dg = np.zeros(itr_max)
        obj = np.zeros(itr_max)
        n = lib().orc_vc_fit(m.h, int(itr_max), int(lbfgs_max), _dptr(dg), _dptr(obj), int(itr_max))
        return dg[:n].copy(), obj[:n].copy()
    finally:
        m.close()

"""TEST INFRASTRUCTURE ONLY: ctypes driver for the reference's own kernels built for the host.

``oracle/_ref/libggplvm_ref.so`` is the unchanged reference source (kernel_funcs.cu,
chol.cu, util_cuda.cu, init.cu, DataFrame.cu, SparseMat.cu and the kernels of
ggplvm.cu) compiled with ``oracle/ref_shim.h`` and driven by ``oracle/ref_harness.cpp``
in the reference driver's call order (ggplvm.cu:951-1354). Only tests, ``smoke()`` and
the CPU legs of ``bench.py`` may load it, as the checker and the CPU baseline.
"""
from __future__ import annotations

import ctypes
import os
import tempfile
from typing import Dict, Optional

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REF_SO = os.path.join(HERE, "_ref", "libggplvm_ref.so")

_dp = ctypes.POINTER(ctypes.c_double)
_ip = ctypes.POINTER(ctypes.c_int)


def available() -> bool:
    return os.path.exists(REF_SO)


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not available():
            raise FileNotFoundError(f"{REF_SO} is not built (make -C oracle ref)")
        L = ctypes.CDLL(REF_SO)
        L.ref_open.restype = ctypes.c_void_p
        L.ref_open.argtypes = [ctypes.c_char_p] * 4 + [ctypes.c_int, ctypes.c_int]
        L.ref_close.argtypes = [ctypes.c_void_p]
        L.ref_dims.argtypes = [ctypes.c_void_p, _ip]
        L.ref_set_params.argtypes = [ctypes.c_void_p] + [_dp] * 6
        L.ref_set_beta.argtypes = [ctypes.c_void_p, _dp]
        for name in ("ref_kernel_mats", "ref_glm_init", "ref_expand_delta", "ref_beta_from_tilde"):
            getattr(L, name).argtypes = [ctypes.c_void_p]
        L.ref_irls_sweep.restype = ctypes.c_double
        L.ref_irls_sweep.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.ref_irls.restype = ctypes.c_int
        L.ref_irls.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.ref_objective_after_irls.restype = ctypes.c_double
        L.ref_objective_after_irls.argtypes = [ctypes.c_void_p, ctypes.c_int]
        L.ref_gradient.argtypes = [ctypes.c_void_p, _dp]
        L.ref_objective.restype = ctypes.c_double
        L.ref_objective.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.ref_lbfgs_update.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]
        L.ref_downdate.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_double, ctypes.c_int]
        L.ref_fit.restype = ctypes.c_int
        L.ref_fit.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, _ip, _dp, ctypes.c_int]
        L.ref_get.restype = ctypes.c_long
        L.ref_get.argtypes = [ctypes.c_void_p, ctypes.c_char_p, _dp]
        L.ref_model_meta.argtypes = [ctypes.c_void_p, _ip, _ip, _ip, _ip]
        L.ref_set_verbose.argtypes = [ctypes.c_int]
        L.ref_score_stats.argtypes = [ctypes.c_void_p, ctypes.c_int, _dp, _dp]
        L.ref_vc_fit.restype = ctypes.c_int
        L.ref_vc_fit.argtypes = [ctypes.c_char_p] * 3 + [ctypes.c_int] * 2 + [_dp] * 5 + [ctypes.c_double] + \
            [ctypes.c_int] * 2 + [_dp, _dp, ctypes.c_int]
        L.ref_de_bfs.restype = ctypes.c_int
        L.ref_de_bfs.argtypes = [ctypes.c_char_p] * 3 + [ctypes.c_int] * 3 + [_dp] * 5 + [ctypes.c_int, _dp, _ip,
                                                                                        _dp, _dp]
        _lib = L
    return _lib


def _ptr(a: Optional[np.ndarray]):
    if a is None:
        return None
    return a.ctypes.data_as(_dp)


class RefModel:
    """One reference context opened from the four input files of the reference CLI."""

    def __init__(self, paths: Dict[str, str], M: int, Q: int):
        L = lib()
        self.h = L.ref_open(paths["Y"].encode(), paths["Z"].encode(), paths["ls"].encode(), paths["Xi"].encode(),
                            int(M), int(Q))
        if not self.h:
            raise IOError("reference could not open its input files")
        d = (ctypes.c_int * 6)()
        L.ref_dims(self.h, d)
        self.N, self.J, self.M, self.P, self.p, self.Q = list(d)
        self._keep = []

    @classmethod
    def from_dataset(cls, ds, workdir: Optional[str] = None) -> "RefModel":
        from gaspacho2_b200.formats import write_dataset

        wd = workdir or tempfile.mkdtemp(prefix="gpl_ref_")
        paths = write_dataset(wd, ds.y, ds.z, ds.ls, ds.X0)
        m = cls(paths, ds.M, ds.Q)
        m.workdir = wd
        return m

    def close(self):
        if self.h:
            lib().ref_close(self.h)
            self.h = None

    def set_params(self, prm) -> None:
        flat = [np.ascontiguousarray(a, dtype=np.float64) for a in prm.flat()]
        self._keep = flat
        lib().ref_set_params(self.h, *[_ptr(a) for a in flat])

    def set_beta(self, beta: np.ndarray) -> None:
        b = np.ascontiguousarray(np.asarray(beta, np.float64).ravel(order="F"))
        lib().ref_set_beta(self.h, _ptr(b))

    def kernel_mats(self):
        lib().ref_kernel_mats(self.h)

    def glm_init(self):
        lib().ref_glm_init(self.h)

    def expand_delta(self):
        lib().ref_expand_delta(self.h)

    def irls_sweep(self, itr: int, jtr: int) -> float:
        return lib().ref_irls_sweep(self.h, itr, jtr)

    def irls(self, itr: int, jtr_max: int) -> int:
        return lib().ref_irls(self.h, itr, jtr_max)

    def objective_after_irls(self, itr: int = 0) -> float:
        return lib().ref_objective_after_irls(self.h, itr)

    def objective(self, itr: int, slot: int) -> float:
        return lib().ref_objective(self.h, itr, slot)

    def gradient(self) -> np.ndarray:
        n = self.N + self.p + self.N * self.Q + self.M * self.Q + self.Q
        g = np.zeros(n)
        lib().ref_gradient(self.h, _ptr(g))
        return g

    def lbfgs_update(self, jtr: int, rhoflag: int):
        lib().ref_lbfgs_update(self.h, jtr, rhoflag)

    def downdate(self, jtr: int, sr: float, rhoflag: int):
        lib().ref_downdate(self.h, jtr, sr, rhoflag)

    def beta_from_tilde(self):
        lib().ref_beta_from_tilde(self.h)

    def fit(self, itr_max: int, lbfgs_budget: int, trace_cap: int = 100000):
        st = (ctypes.c_int * 4)()
        tr = np.zeros(trace_cap)
        rc = lib().ref_fit(self.h, itr_max, lbfgs_budget, st, _ptr(tr), trace_cap)
        stats = dict(outer=st[0], irls=st[1], lbfgs=st[2], evals=st[3])
        ntr = stats["outer"] + stats["lbfgs"]
        return rc, stats, tr[:ntr].copy()

    def get(self, name: str) -> np.ndarray:
        n = lib().ref_get(self.h, name.encode(), None)
        if n < 0:
            raise KeyError(name)
        out = np.zeros(n)
        lib().ref_get(self.h, name.encode(), _ptr(out))
        return out

    def score_stats(self, G: np.ndarray) -> np.ndarray:
        """getScoreStats (ggplvm_de.cu:489-535): G is N x L, the result J x L."""
        G = np.asfortranarray(G, dtype=np.float64)
        L = G.shape[1]
        S = np.zeros(self.J * L)
        lib().ref_score_stats(self.h, L, _ptr(G.ravel(order="F")), _ptr(S))
        return S.reshape(L, self.J).T

    def model_meta(self):
        nh = (ctypes.c_int * (self.p + 1))()
        mc = (ctypes.c_int * self.P)()
        mv = (ctypes.c_int * self.P)()
        mk = (ctypes.c_int * self.P)()
        lib().ref_model_meta(self.h, nh, mc, mv, mk)
        return np.array(nh), np.array(mc), np.array(mv), np.array(mk)


def de_bfs(ds, prm, Mredc: int, Mfull: int, jtr_max: int = 1000, workdir: Optional[str] = None):
    """The reference's own DE model comparison (ggplvm_de.cu:886-1207, through ref_de_bfs)
    on the dataset's files at prm's fitted Omega, delta, X, T (Mfull x Q) and rho.
    Returns (BFs J x (Q + 2), sweeps per model, full-model beta P x J, phi)."""
    from gaspacho2_b200.formats import write_dataset

    wd = workdir or tempfile.mkdtemp(prefix="gpl_ref_de_")
    paths = write_dataset(wd, ds.y, ds.z, ds.ls, ds.X0)
    Q, J = ds.Q, ds.J
    arr = [np.ascontiguousarray(np.asarray(a, np.float64).ravel(order="F"))
           for a in (prm.Omega, prm.delta, prm.X, prm.T, prm.rho)]
    BFs = np.zeros(J * (Q + 2))
    sweeps = (ctypes.c_int * (Q + 2))()
    P1 = 1 + int(sum(int(c) * int(v) for c, v in zip(ds.z.c, ds.z.v))) + int(Mfull)  # nh[p] (DataFrame.cu:77-89)
    beta = np.zeros(P1 * J)
    phi = np.zeros(J)
    P1r = lib().ref_de_bfs(paths["Y"].encode(), paths["Z"].encode(), paths["ls"].encode(), Q, int(Mredc), int(Mfull),
                           *[_ptr(a) for a in arr], int(jtr_max), _ptr(BFs), sweeps, _ptr(beta), _ptr(phi))
    if P1r < 0:
        raise IOError("reference could not open its input files")
    return BFs.reshape(Q + 2, J).T.copy(), list(sweeps), beta[:P1r * J].reshape(J, P1r).T.copy(), phi


def vc_fit(ds, prm, init_dg: float = 0.01, itr_max: int = 100, lbfgs_max: int = 100,
           workdir: Optional[str] = None):
    """The reference's own variance-component driver (ggplvm_delta.cu:784-1097, through
    ref_vc_fit) on the dataset's files; ``prm`` as for oracle.port.vc_fit. Returns (delta[p-2]
    after each outer iteration, the objective after each outer iteration)."""
    from gaspacho2_b200.formats import write_dataset

    wd = workdir or tempfile.mkdtemp(prefix="gpl_ref_vc_")
    paths = write_dataset(wd, ds.y, ds.z, ds.ls, ds.X0)
    arr = [np.ascontiguousarray(np.asarray(a, np.float64).ravel(order="F"))
           for a in (prm.Omega, prm.delta, prm.X, prm.T, prm.rho)]
    dg = np.zeros(itr_max)
    obj = np.zeros(itr_max)
    n = lib().ref_vc_fit(paths["Y"].encode(), paths["Z"].encode(), paths["ls"].encode(), int(ds.M), int(ds.Q),
                         *[_ptr(a) for a in arr], float(init_dg), int(itr_max), int(lbfgs_max), _ptr(dg), _ptr(obj),
                         int(itr_max))
    if n < 0:
        raise IOError("reference could not open its input files")
    return dg[:n].copy(), obj[:n].copy()

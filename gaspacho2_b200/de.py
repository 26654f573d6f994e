"""The differential-expression driver's model comparison over the C ABI (ggplvm_de.cu).

After a fit, the reference's DE driver (``ggplvm_de``, ggplvm_de.cu:886-1237) refits the GLM
part by IRLS at the fitted Omega, delta, X and rho for

  * the null model Z0, without the GP (ggplvm_de.cu:1067-1107),
  * one model per latent dimension q, the GP over dimension q alone with ``Mredc``
    equispaced inducing points (ggplvm_de.cu:1110-1133, reduced branch),
  * the full model, the GP over all dimensions with the fitted ``Mfull`` inducing points
    (ggplvm_de.cu:1112-1119),

and keeps each model's per-gene log-likelihood in the J x (Q + 2) table it writes to
``BFs_de.gz``. ``de_bfs`` runs the same sequence on three contexts (null, reduced, full):
phi starts at 1 and each model starts from the previous model's final phi, as in the
reference; the null model's tolerance is 1e-5 and the others' 1e-8.
"""
from __future__ import annotations

from typing import Dict, List, Optional

import numpy as np

from . import _lib
from .model import GPLVM


def ta_equispaced(M: int, Q: int) -> np.ndarray:
    """initTaEquispaced (util.c:57-71): the reduced models' M x Q inducing points."""
    T = np.zeros(M * Q)
    _lib.load().gpl_ta_equispaced(int(M), int(Q), T.ctypes.data_as(_lib._dp))
    return T.reshape(Q, M).T.copy()


def open_contexts(y, z, ls, X, Q: int, Mredc: int, Mfull: int, device: int = 0, stream: Optional[int] = None):
    """The three contexts of a model comparison: (null, per-dimension, full). The null model's
    one-column GP block is held inert (Knm = 0), standing in for the GP-free design Z0."""
    out = []
    try:
        for M in (1, Mredc, Mfull):
            out.append(GPLVM(y, z, ls, X, M, Q, device=device, stream=stream))
    except Exception:
        for m in out:
            m.close()
        raise
    return tuple(out)


def de_bfs(y, z, ls, prm, Q: int, Mredc: int, Mfull: int, jtr_max: int = 1000, device: int = 0,
           stream: Optional[int] = None, keep_models: bool = False, contexts=None) -> Dict:
    """The DE driver's model table at the fitted parameters ``prm`` (Omega, delta, X, T of
    Mfull x Q inducing points, rho; its phi is not used: the driver restarts phi at 1).

    Returns a dict with ``BFs`` (J x (Q + 2): null, dimensions 0..Q-1, full), ``sweeps`` per
    model, ``phi`` after the full model, and ``full`` (the full model's context, left open
    for score statistics). ``contexts`` (from ``open_contexts``) are used as given and left
    open; otherwise the null and per-dimension contexts are closed here and the caller closes
    ``full``. With ``keep_models``, ``betas`` and ``kmats`` hold each model's coefficients
    (P x J) and (Knm, Kmm), as the reference appends them to Beta_de.gz and Knm_de.gz."""
    N = int(np.asarray(ls).shape[0])
    J = int(y.J)
    BFs = np.zeros((J, Q + 2))
    sweeps: List[int] = []
    betas, kmats = [], []
    phi = np.ones(J)
    X = np.asarray(prm.X, np.float64)
    Omega = np.asarray(prm.Omega, np.float64)
    delta = np.asarray(prm.delta, np.float64)
    rho = np.asarray(prm.rho, np.float64)
    from .formats import Params

    def run(m: GPLVM, model, T, tol, col):
        nonlocal phi
        m.set_params(Params(Omega, delta, X, np.asarray(T, np.float64).reshape(m.M, Q), rho, phi.copy()))
        m.de_model(model)
        lk, n, _ = m.de_irls(jtr_max, tol)
        BFs[:, col] = lk
        sweeps.append(n)
        phi = m.get("phi").copy()
        if keep_models:
            betas.append(m.get("Beta").reshape(J, m.P).T.copy())
            kmats.append((m.get("Knm").reshape(m.M, N).T.copy(), m.get("Kmm").reshape(m.M, m.M).T.copy()))

    own = contexts is None
    m0, mr, mf = contexts if contexts is not None else open_contexts(y, z, ls, X, Q, Mredc, Mfull, device, stream)
    try:
        run(m0, "null", np.zeros((1, Q)), 1e-5, 0)
        Tr = ta_equispaced(Mredc, Q)
        for q in range(Q):
            run(mr, q, Tr, 1e-8, q + 1)
        run(mf, "full", np.asarray(prm.T, np.float64), 1e-8, Q + 1)
    except Exception:
        if own:
            for m in (m0, mr, mf):
                m.close()
        raise
    if own:
        m0.close()
        mr.close()
    out = dict(BFs=BFs, sweeps=sweeps, phi=phi, full=mf)
    if keep_models:
        out.update(betas=betas, kmats=kmats)
    return out

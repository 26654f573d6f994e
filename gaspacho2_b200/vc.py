"""The variance-component driver over the C ABI (ggplvm_delta.cu:784-1097).

The reference's ``ggplvm_delta`` (whose main does not compile as shipped) refits one prior
variance, delta[p-2], of a design whose last variable is the one of interest (a genotype), at
a previous fit's Omega, X, T and rho: IRLS phases in the DE driver's forms alternate with
L-BFGS on log delta[p-2]. It reads params.bin with the p - 1 deltas of the fit (the design
without that variable), starts delta[p-2] at --init-deltaG and leaves delta[p-1], the GP's,
at initParams' 0.3; ``vc_fit`` sets the parameters the same way.
"""
from __future__ import annotations

from typing import Optional

import numpy as np

from .formats import Params
from .model import GPLVM

INIT_DELTA_GP = 0.3  # initParams (init.cu:27-48): the value delta[p-1] keeps in the driver


def vc_fit(y, z, ls, prm, M: int, Q: int, init_dg: float = 0.01, itr_max: int = 100, lbfgs_max: int = 100,
           device: int = 0, stream: Optional[int] = None):
    """``z`` ends with the variable whose variance is refitted; ``prm`` holds the fit's Omega,
    X, T (M x Q), rho and its p - 1 deltas. Returns (delta[p-2], objective) after each outer
    iteration."""
    with GPLVM(y, z, ls, prm.X, M, Q, device=device, stream=stream) as m:
        p = m.p
        d = np.empty(p)
        d[:p - 2] = np.asarray(prm.delta, np.float64)[:p - 2]
        d[p - 2] = init_dg
        d[p - 1] = INIT_DELTA_GP
        m.set_params(Params(np.asarray(prm.Omega, np.float64), d, np.asarray(prm.X, np.float64),
                            np.asarray(prm.T, np.float64).reshape(M, Q), np.asarray(prm.rho, np.float64),
                            np.ones(int(y.J))))
        return m.vc_fit(itr_max, lbfgs_max)

"""The gradient of the fit (getGradLogOmega, getGradLogDelta, getGradTau, getGradLogRho,
ggplvm.cu:46-376) is the exact derivative of the line-search objective (getLkhd + collectLkhd,
ggplvm.cu:703-815) at the IRLS's fixed W and nu: a central difference of the oracle's objective
along a random direction of each parameter block (log Omega, log delta, X, T, log rho) matches
the gradient's projection on it. The oracle is pinned bit for bit to the reference's kernels
(test_oracle_golden.py), so this is a property of the reference's formulas, independent of the
problem size."""
import numpy as np
import pytest

from gaspacho2_b200.formats import Params
from oracle import port
from tests import golden_util as gu

H = 1e-4     # step in the parameters' own coordinates (log scale for Omega, delta, rho)
TOL = 1e-5   # |fd - g.d| <= TOL * |g_block| |d|: truncation O(h^2) plus rounding of the objective


@pytest.mark.parametrize("name", gu.CASES)
def test_gradient_is_the_objectives_derivative(name):
    gd = gu.load(name)
    o = port.OracleModel.from_dataset(gd)
    o.set_params(gd.init)
    o.kernel_mats()
    o.glm_init()
    o.irls(0, 200)
    o.objective_after_irls(0)
    g = o.gradient()
    N, p, Q, M = o.N, o.p, o.Q, o.M
    Om, de, X, T, rho, phi = (o.get(k) for k in ("Omega", "delta", "X", "T", "rho", "phi"))
    ends = np.cumsum([0, N, p, N * Q, M * Q, Q])
    assert ends[-1] == g.size
    blocks = dict(zip(("log Omega", "log delta", "X", "T", "log rho"), zip(ends[:-1], ends[1:])))

    def objective_at(v):
        b = {k: v[a:e] for k, (a, e) in blocks.items()}
        o.set_params(Params(Om * np.exp(b["log Omega"]), de * np.exp(b["log delta"]), X + b["X"], T + b["T"],
                            rho * np.exp(b["log rho"]), phi))
        return o.objective(0, 1)

    rng = np.random.default_rng(7)
    for blk, (a, e) in blocks.items():
        d = np.zeros(g.size)
        d[a:e] = rng.standard_normal(e - a)
        fd = (objective_at(H * d) - objective_at(-H * d)) / (2 * H)
        gd_ = float(g @ d)
        scale = np.linalg.norm(g[a:e]) * np.linalg.norm(d)
        assert abs(fd - gd_) <= TOL * scale, f"{name} {blk}: fd {fd:.10e} vs g.d {gd_:.10e} (scale {scale:.3e})"
    o.close()

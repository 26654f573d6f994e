"""The batched form on the GPU: the persistent per-gene IRLS tail, evaluations as CUDA graphs,
the autotuner, and the bounded device wait.

Each of the three changes only how the same kernels are scheduled (one persistent launch over a
gene queue instead of four launches; graph replay instead of per-kernel launches; which CTA
takes which tile), so each is checked for the SAME BITS as the plain path on the same inputs,
at the benchmark's shape (tests/golden/c2_head.npz: M = 128, Q = 10, P = 236) and on a fixture
with count-handling edge cases (an all-zero gene, an all-nonzero gene, out-of-order indices)."""
import numpy as np
import pytest

from gaspacho2_b200 import GPLVM
from tests import golden_util as gu

pytestmark = pytest.mark.gpu


def _irls_state(gd, **opts):
    with GPLVM.from_dataset(gd) as m:
        for k, v in opts.items():
            m.set_option(k, v)
        m.set_params(gd.init)
        m.kernel_mats()
        m.glm_init()
        lk = [m.irls_sweep(0, j) for j in range(3)]
        out = {k: m.get(k) for k in ("Beta", "phi", "lkhds", "Psi")}
        out["sweeps"] = np.array(lk)
        out["obj"] = np.array([m.objective_after_irls(0)])
        out["grad"] = m.gradient()
        out["tBeta"] = m.get("tBeta")
    return out


@pytest.mark.parametrize("name", ["c2_head", "edges"])
def test_fused_tail_same_bits(name):
    gd = gu.load(name)
    a = _irls_state(gd)
    b = _irls_state(gd, fused_tail=1)
    c = _irls_state(gd, fused_tail=1, tail_ctas_per_sm=1)
    for k in a:
        assert np.array_equal(a[k], b[k], equal_nan=True), f"{k}: fused tail differs"
        assert np.array_equal(a[k], c[k], equal_nan=True), f"{k}: fused tail (1 CTA/SM) differs"


def _fit(gd, budget=12, **opts):
    with GPLVM.from_dataset(gd) as m:
        for k, v in opts.items():
            m.set_option(k, v)
        m.set_params(gd.init)
        m.kernel_mats()
        m.glm_init()
        rc, st, tr = m.fit(1, budget)
        out = {k: m.get(k) for k in ("Omega", "delta", "X", "T", "rho", "phi", "Beta")}
        out["trace"] = tr
        out["stats"] = np.array([st["outer"], st["irls"], st["lbfgs"], st["evals"]])
        info = {k: m.get_option(k) for k in ("graph", "graph_replays", "autotune")}
        tun = {k: m.tuning(k) for k in ("pair_gram", "pair_v", "irls_tail", "eta_tile")}
    return out, info, tun


@pytest.mark.parametrize("name", ["c0_small", "c2_head"])
def test_graph_fit_same_bits(name):
    """The budgeted fit with every objective and gradient replayed from captured graphs (and the
    fused tail) against the plain launches: the same trace, decisions and parameters, bit for
    bit; the graphs were replayed."""
    gd = gu.load(name)
    a, _, _ = _fit(gd)
    b, info, _ = _fit(gd, graph=1, fused_tail=1)
    assert info["graph"] == 1, "graph capture was refused"
    assert info["graph_replays"] >= 10
    for k in a:
        assert np.array_equal(a[k], b[k]), f"{k}: graph replay differs"


def test_autotuned_fit_same_bits_and_records():
    """The autotuner times every candidate on the fit's own launches and settles: the fit's
    results are the plain fit's bits, and every choice that came up holds a chosen value and a
    measured time for each candidate."""
    gd = gu.load("c2_head")
    a, _, _ = _fit(gd)
    b, info, tun = _fit(gd, autotune=1, graph=1, fused_tail=1)
    for k in a:
        assert np.array_equal(a[k], b[k]), f"{k}: autotuned fit differs"
    for name in ("pair_gram", "irls_tail", "pair_v", "eta_tile"):
        t = tun[name]
        assert t["chosen"] is not None, f"{name}: never settled"
        assert t["chosen"] in t["candidates_ms"]
        assert all(v is None or v > 0 for v in t["candidates_ms"].values())
    assert info["graph"] == 1 and info["graph_replays"] > 0


def test_evaluate_device_graph_replay():
    """gpl_evaluate through graphs equals the eager evaluation at the same parameters, on the
    first call (eager, then captured) and on replays."""
    gd = gu.load("c2_head")
    with GPLVM.from_dataset(gd) as m:
        m.set_params(gd.init)
        m.kernel_mats()
        m.glm_init()
        m.irls(0, 5)
        m.objective_after_irls(0)
        x = m.params_vector()
        v0, g0 = m.evaluate(x)
        g0 = g0.copy()
        m.set_option("graph", 1)
        for _ in range(3):
            v, g = m.evaluate(x)
            assert v == v0
            assert np.array_equal(g, g0)
        assert m.get_option("graph_replays") >= 4


def test_bounded_wait_runs_out_and_context_survives():
    """Failure detection of the device waits: the bounded wait the tensor-core kernels use, run
    against a barrier that nothing completes, gives up after its limit and is reported as
    GPL_ERR_TIMEOUT; the same context then evaluates normally."""
    import time

    from gaspacho2_b200 import _lib

    gd = gu.load("c0_small")
    with GPLVM.from_dataset(gd) as m:
        L = _lib.load()
        t0 = time.time()
        rc = L.gpl_wait_probe(m.h, 20_000_000)  # 20 ms
        dt = time.time() - t0
        assert _lib.ERRORS.get(rc) == "GPL_ERR_TIMEOUT", rc
        assert 0.015 < dt < 5.0
        assert b"gave up" in L.gpl_last_error(m.h)
        m.set_params(gd.init)
        m.kernel_mats()
        m.glm_init()
        v = m.irls_sweep(0, 0)
        assert np.isfinite(v)
        assert np.isclose(v, float(gd.g["sweep0_lkhd"]), rtol=1e-10)

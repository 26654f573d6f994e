"""The precision form (GPL_PREC_BF16X3) against the plain FP64 path, through the C ABI.

The precision form runs the Gram and the gradient contraction on tcgen05 tensor cores (BF16
hi/lo products, FP32 runs folded into FP64 in TMEM) over the dense columns whitened by the
prior's Cholesky factor, maps the results back in FP64 and refines every per-gene solve against
the FP64 operator; everything else stays FP64. Bars, per objective+gradient
evaluation at the same state:
  * every per-gene Cholesky succeeds (the whitening is what makes this hold: without it,
    1e-6 Gram errors against cond(Psi_j) ~ 1e14 fail the factorisation);
  * the objective within 1e-6 relative of FP64 (measured ~1e-9 after the refinement of the
    solve that enters it);
  * the gradient blocks for Omega, delta, X and rho within 2e-3 (relative L2), T within 5e-2
    (measured up to 1.2e-5 and 4.4e-4), except at config 0, whose cond(Kmm) = 3.5e10 makes even the
    FP64 path's gradient move by 5e-5 under a change of summation order; there only finiteness
    is required."""
import numpy as np
import pytest

from gaspacho2_b200 import GPLVM, synth

pytestmark = pytest.mark.gpu


def _evaluate(ds, precision):
    with GPLVM.from_dataset(ds, precision="fp64") as m:
        m.set_params(ds.init)
        m.kernel_mats()
        m.glm_init()
        for j in range(3):
            m.irls_sweep(0, j)
        m.objective_after_irls(0)
        m.set_precision(precision)
        v, g = m.evaluate(m.params_vector())
        P = m.P
        psi = m.get("Psi").reshape(m.J, P, P)
        failed = sum(1 for x in psi if np.abs(np.diag(x)).max() == 0)
        return v, g.copy(), failed, (m.N, m.Q, m.M)


def _blocks(g, dims):
    N, Q, M = dims
    p = len(g) - N - N * Q - M * Q - Q
    out, off = {}, 0
    for name, n in (("Omega", N), ("delta", p), ("X", N * Q), ("T", M * Q), ("rho", Q)):
        out[name] = g[off:off + n]
        off += n
    return out


@pytest.mark.parametrize("cfg,kw", [(0, dict(G=100)), (1, dict(N=6000, G=300)),
                                    (2, dict(N=6000, G=200, M=64, Q=5))])
def test_precision_form_against_fp64(cfg, kw):
    ds = synth.make(cfg, 5, init=True, **kw)
    v0, g0, f0, dims = _evaluate(ds, "fp64")
    v1, g1, f1, _ = _evaluate(ds, "bf16x3")
    assert f0 == 0 and f1 == 0, (f0, f1)
    rel = abs(v1 - v0) / abs(v0)
    print(f"config {cfg}: objective rel err {rel:.2e}")
    assert rel <= 1e-6
    assert np.all(np.isfinite(g1))
    b0, b1 = _blocks(g0, dims), _blocks(g1, dims)
    bad = []
    for name in b0:
        e = np.linalg.norm(b1[name] - b0[name]) / max(np.linalg.norm(b0[name]), 1e-300)
        tol = 5e-2 if name == "T" else 2e-3
        print(f"  grad {name:5s} rel-l2 {e:.2e} (tol {tol:.0e})")
        if cfg != 0 and not e <= tol:
            bad.append(f"{name}: {e:.2e}")
    assert not bad, bad


@pytest.mark.parametrize("name", ["c2_head", "c2_cats"])
def test_precision_form_against_reference_golden(name):
    """The precision form's phases against the reference's own kernels (the golden vectors, FP64
    on the host): at the benchmark's model shape (c2_head: M = 128, Q = 10, P = 236) and with an
    empty donor level (c2_cats). The objective values within 1e-6 relative, the gradient blocks
    within 1e-4 (T within 1e-3) relative L2 (measured: objective 4.7e-9 and 3.8e-8, gradient
    blocks 7.4e-8 to 4.3e-6, T 9.3e-6 and 2.5e-5)."""
    from tests import golden_util as gu

    gd = gu.load(name)
    with GPLVM.from_dataset(gd, precision="bf16x3") as m:
        out = gu.run_phases(m, gd)
        dims = (m.N, m.Q, m.M)
    ref = gd.g
    bad = []
    for k in ("sweep0_lkhd", "obj0", "obj1"):
        a, b = float(np.ravel(out[k])[0]), float(np.ravel(ref[k])[0])
        e = abs(a - b) / abs(b)
        print(f"{name}: {k} rel err {e:.2e}")
        if not e <= 1e-6:
            bad.append(f"{k}: {e:.2e}")
    b0, b1 = _blocks(np.asarray(ref["grad0"]), dims), _blocks(np.asarray(out["grad0"]), dims)
    for blk in b0:
        e = np.linalg.norm(b1[blk] - b0[blk]) / max(np.linalg.norm(b0[blk]), 1e-300)
        tol = 1e-3 if blk == "T" else 1e-4
        print(f"{name}: grad {blk:5s} rel-l2 {e:.2e} (tol {tol:.0e})")
        if not e <= tol:
            bad.append(f"grad {blk}: {e:.2e}")
    assert not bad, bad


def _evaluate_opts(ds, opts):
    with GPLVM.from_dataset(ds, precision="fp64") as m:
        for k, v in opts.items():
            m.set_option(k, v)
        m.set_params(ds.init)
        m.kernel_mats()
        m.glm_init()
        for j in range(3):
            m.irls_sweep(0, j)
        m.objective_after_irls(0)
        m.set_precision("bf16x3")
        v, g = m.evaluate(m.params_vector())
        return v, g.copy()


@pytest.mark.parametrize("cfg,kw", [(1, dict(N=6000, G=300)), (2, dict(N=6000, G=200, M=64, Q=5))])
def test_cta_pair_contractions(cfg, kw):
    """Option tc_pair (the Gram and the gradient contraction on CTA pairs: one M = 256
    tcgen05.mma.cta_group::2 per K step over two CTAs' shared memory) against the single-CTA
    kernel: the same products in the same K order per output, so the objective within 1e-12 and
    the gradient within 1e-9 (relative). Both cases have 68 dense columns, 2,346 pairs in 19 tiles:
    the odd CTA of the last pair has no pairs (its A rows lie past the matrix and load as zeros)."""
    ds = synth.make(cfg, 6, init=True, **kw)
    v0, g0 = _evaluate_opts(ds, {})
    v1, g1 = _evaluate_opts(ds, {"tc_pair": 1})
    rel = abs(v1 - v0) / abs(v0)
    gr = np.linalg.norm(g1 - g0) / np.linalg.norm(g0)
    print(f"config {cfg}: objective {rel:.2e}, gradient {gr:.2e}, bitwise {v1 == v0 and np.array_equal(g1, g0)}")
    assert rel <= 1e-12
    assert gr <= 1e-9


def test_logdet_probe_and_fp64_line_search():
    """The precision form's objective with the log-determinant probe (default) against FP64 at the
    same state within 1e-6, and a budgeted fit with option ls_fp64 (a failed line search repeated
    with the FP64 objective) that ends finite with the precision form restored."""
    ds = synth.make(2, 8, init=True, N=6000, G=200, M=64, Q=5)
    v0, _ = _evaluate_opts(ds, {"logdet_probe": 0})
    v1, _ = _evaluate_opts(ds, {})
    with GPLVM.from_dataset(ds, precision="fp64") as m:
        m.set_params(ds.init)
        m.kernel_mats()
        m.glm_init()
        for j in range(3):
            m.irls_sweep(0, j)
        m.objective_after_irls(0)
        vf, _ = m.evaluate(m.params_vector())
    print(f"objective vs FP64: probe {abs(v1 - vf) / abs(vf):.2e}, without {abs(v0 - vf) / abs(vf):.2e}")
    assert abs(v1 - vf) / abs(vf) <= 1e-6
    with GPLVM.from_dataset(ds, precision="bf16x3") as m:
        m.set_option("ls_fp64", 1)
        m.set_params(ds.init)
        m.kernel_mats()
        m.glm_init()
        rc, st, tr = m.fit(3, 40)
        print(f"fit: {st}, repeated steps {m.get_option('ls_fp64_steps')}, last {tr[-1]:.6e}")
        assert np.all(np.isfinite(tr))
        assert m.get_option("ls_fp64_steps") >= 0

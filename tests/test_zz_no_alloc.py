"""gpl_kernel_mats_noalloc: the allocation-free entry point against the context-based one.

Callers that cannot allocate device memory (work enqueued under stream capture, real-time
loops, plugins whose framework owns the memory) pass their own device buffers; the only
scratch, the M x M Kmm factor, is a fixed array inside the library. This file is collected
last so a failure here never hides the other tests.
"""
import ctypes

import numpy as np
import pytest

from gaspacho2_b200 import GPLVM, _lib
from tests import golden_util as gu

pytestmark = pytest.mark.gpu

TOL = 1e-12  # the same kernels in the same order as gpl_kernel_mats: equal to rounding


def _through_context(gd):
    with GPLVM.from_dataset(gd) as m:
        m.set_params(gd.init)
        m.kernel_mats()
        N, M = m.N, m.M
        knm = m.get("Knm").reshape(M, N).T
        kk = m.get("KinvKmn").reshape(N, M)
        tits = m.get("titsias")
    return knm, kk, tits


def _without_allocation(torch, gd, M_override=None):
    """Device buffers come from torch here (the test may allocate; the entry point may not).
    Outputs start as NaN so any element the call fails to write shows up."""
    N, Q = gd.N, gd.Q
    M = gd.M if M_override is None else M_override
    dev = dict(dtype=torch.float64, device="cuda")
    X = torch.tensor(np.asarray(gd.init.X, np.float64).ravel(order="F"), **dev)
    T = torch.tensor(np.asarray(gd.init.T, np.float64).ravel(order="F"), **dev)
    rho = torch.tensor(np.asarray(gd.init.rho, np.float64), **dev)
    knm = torch.full((N * max(M, 1),), float("nan"), **dev)
    kk = torch.full((N * max(M, 1),), float("nan"), **dev)
    tits = torch.full((N,), float("nan"), **dev)
    torch.cuda.synchronize()
    L = _lib.load()
    p = lambda t: ctypes.c_void_p(t.data_ptr())  # noqa: E731
    rc = L.gpl_kernel_mats_noalloc(N, M, Q, p(X), p(T), p(rho), p(knm), p(kk), p(tits), None)
    torch.cuda.synchronize()
    out = (knm.cpu().numpy(), kk.cpu().numpy(), tits.cpu().numpy())
    if rc != 0:
        return rc, out
    return rc, (out[0].reshape(M, N).T, out[1].reshape(M, N).T, out[2])


def test_noalloc_matches_context_path_on_consecutive_calls():
    torch = pytest.importorskip("torch")
    cases = [gu.load("c0_small"), gu.load("c2_cats"), gu.load("c0_small")]
    for gd in cases:  # different M in a row: the shared work array keeps the last call's data
        ref = _through_context(gd)
        rc, got = _without_allocation(torch, gd)
        assert rc == 0, _lib.ERRORS.get(rc, rc)
        for name, a, b in zip(("Knm", "KinvKmn", "titsias"), got, ref):
            assert np.all(np.isfinite(a)), f"{name}: unwritten elements"
            e = gu.rel_err(a, b)
            assert e <= TOL, f"{name}: rel err {e:.3e}"


def test_noalloc_fills_the_whole_scratch_at_its_limit():
    """M = GPL_NOALLOC_MAX_M uses every element of the fixed 256 x 256 array; twice in a row,
    after a smaller M left other contents in it."""
    torch = pytest.importorskip("torch")
    from gaspacho2_b200 import synth

    import dataclasses

    gd = synth.make(2, 3, N=700, G=12, M=256, Q=10)
    # 256 inducing points spread wide (N(0, 4 I) in 10 dimensions) keep Kmm well conditioned; k-means
    # centres of 700 cells would nearly coincide and make its factor fail in both paths
    T = 2.0 * np.random.default_rng(5).standard_normal((256, 10))
    gd = dataclasses.replace(gd, init=dataclasses.replace(gd.init, T=T))
    ref = _through_context(gd)
    assert np.all(np.isfinite(ref[1])), "the context path's Kmm^-1 k_n must be finite for this case"
    for _ in range(2):
        rc, got = _without_allocation(torch, gd)
        assert rc == 0, _lib.ERRORS.get(rc, rc)
        for name, a, b in zip(("Knm", "KinvKmn", "titsias"), got, ref):
            assert np.all(np.isfinite(a)), f"{name}: unwritten or non-finite elements"
            e = gu.rel_err(a, b)
            assert e <= TOL, f"{name}: rel err {e:.3e}"
        small = gu.load("c0_small")
        rc, _ = _without_allocation(torch, small)
        assert rc == 0


def test_noalloc_rejects_m_beyond_its_fixed_scratch():
    torch = pytest.importorskip("torch")
    gd = gu.load("c0_small")
    limit = 256
    rc, out = _without_allocation(torch, gd, M_override=limit + 1)
    assert _lib.ERRORS.get(rc) == "GPL_ERR_LIMIT"
    assert np.all(np.isnan(out[2])), "a refused call must not write its outputs"

"""The variance-component driver (ggplvm_delta.cu:784-1097) on the oracle: the C restatement
against the trajectories produced by the reference's own kernels (tests/golden/vc_c1.npz;
the reference's main does not compile, its kernels do), and against the live reference
build when present."""
import numpy as np
import pytest

from gaspacho2_b200 import synth
from oracle import port, refcpu
from tests import golden_util as gu

TOL = 1e-12  # the same arithmetic in the same order


@pytest.mark.parametrize("tag,it", [("i3", 3), ("i8", 8)])
def test_oracle_vc_matches_golden(tag, it):
    ds, prm = gu.load_vc("vc_c1")
    dg, obj = port.vc_fit(ds, prm, float(ds.g["in_init_dg"]), it, 100)
    assert dg.shape[0] == it
    assert gu.rel_err(dg, ds.g[f"vc_{tag}_dg"]) <= TOL
    assert gu.rel_err(obj, ds.g[f"vc_{tag}_obj"]) <= TOL


@pytest.mark.skipif(not refcpu.available(), reason="reference host build not present")
def test_oracle_vc_matches_live_reference():
    import dataclasses

    from gaspacho2_b200.formats import Design

    ds = synth.make(1, 12, init=True, N=200, G=16, M=6, Q=2)
    rng = np.random.default_rng(3)
    g = rng.binomial(2, 0.4, size=(ds.N, 1)).astype(np.float64)
    z = ds.z
    ds = dataclasses.replace(ds, z=Design(z.N, np.append(z.c, 1).astype(np.int32), np.append(z.v, 1).astype(np.int32),
                                          list(z.columns) + [g]))
    a = refcpu.vc_fit(ds, ds.init, 0.05, 3, 20)
    b = port.vc_fit(ds, ds.init, 0.05, 3, 20)
    assert gu.rel_err(b[0], a[0]) <= TOL and gu.rel_err(b[1], a[1]) <= TOL

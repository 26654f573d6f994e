"""The DE driver's model comparison (ggplvm_de.cu:886-1207) on the oracle: the C restatement
against the golden tables produced by the reference's own kernels (tests/golden/de_*.npz),
and against the live reference build on a fresh seeded case when that build is present."""
import numpy as np
import pytest

from gaspacho2_b200 import synth
from oracle import port, refcpu
from tests import golden_util as gu

TOL = 1e-12  # the same arithmetic in the same order


@pytest.fixture(scope="module", params=gu.DE_CASES)
def case(request):
    return gu.load(request.param)


@pytest.mark.parametrize("tag,jt", [("j3", 3), ("conv", 1000)])
def test_oracle_de_bfs_matches_golden(case, tag, jt):
    g = case.g
    bfs, sweeps, beta, phi = port.de_bfs(case, case.init, int(g["in_Mredc"]), case.M, jt)
    assert sweeps == g[f"de_{tag}_sweeps"].tolist()
    assert gu.rel_err(bfs, g[f"de_{tag}_BFs"]) <= TOL
    assert gu.rel_err(phi, g[f"de_{tag}_phi"]) <= TOL
    assert gu.rel_err(beta, g[f"de_{tag}_beta_full"]) <= TOL


def test_null_model_loader_value():
    """The reference's loader leaves 199.0 in the first cell of the last design variable of a
    GP-free design (DataFrame.cu:112-113, 131). Setting that cell to 199.0 in the input
    therefore leaves the null model's column unchanged while the GP models, which see the
    loaded value, change."""
    import copy
    gd = gu.load("de_c1")
    assert gd.z.c[-1] == 1
    gd2 = copy.deepcopy(gd)
    gd2.z.columns[-1] = gd2.z.columns[-1].copy()
    gd2.z.columns[-1].reshape(-1)[0] = 199.0
    a = port.de_bfs(gd, gd.init, int(gd.g["in_Mredc"]), gd.M, 3)[0]
    b = port.de_bfs(gd2, gd2.init, int(gd2.g["in_Mredc"]), gd2.M, 3)[0]
    assert np.array_equal(a[:, 0], b[:, 0])
    assert not np.allclose(a[:, -1], b[:, -1])


def test_ta_equispaced():
    """initTaEquispaced (util.c:57-71)."""
    T = port.ta_equispaced(4, 3)
    assert np.allclose(T[:, 0], np.arange(1, 5) / 5 * 2 * 3.14159265358979)
    assert np.allclose(T[:, 1], (np.arange(1, 5) / 5 - 0.5) * 6.0)
    assert np.array_equal(T[:, 1], T[:, 2])


@pytest.mark.skipif(not refcpu.available(), reason="reference host build not present")
def test_oracle_de_bfs_matches_live_reference():
    ds = synth.make(1, 11, init=True, N=200, G=16, M=6, Q=2)
    a = refcpu.de_bfs(ds, ds.init, 3, ds.M, 8)
    b = port.de_bfs(ds, ds.init, 3, ds.M, 8)
    assert a[1] == b[1]
    for x, y in zip((a[0], a[2], a[3]), (b[0], b[2], b[3])):
        assert gu.rel_err(y, x) <= TOL

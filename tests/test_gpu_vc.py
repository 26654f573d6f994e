"""The variance-component driver on the GPU, through the C ABI (gpl_vc_fit), against the
trajectories of the reference's own kernels (tests/golden/vc_c1.npz): delta[p-2] and the
objective after each outer iteration. Each outer iteration's IRLS phase, Gram, factorisations
and Laplace objective run on the DMMA kernels in an order of summation other than the
reference's loops; the line search's discrete decisions then see the same comparisons.
Bars: delta[p-2] within 1e-9 and the objective within 1e-9 relative after every outer
iteration."""
import numpy as np
import pytest

from gaspacho2_b200 import GPLVM, vc
from gaspacho2_b200._lib import GplError
from tests import golden_util as gu

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("tag,it", [("i3", 3), ("i8", 8)])
def test_vc_matches_reference(tag, it):
    ds, prm = gu.load_vc("vc_c1")
    dg, obj = vc.vc_fit(ds.y, ds.z, ds.ls, prm, ds.M, ds.Q, float(ds.g["in_init_dg"]), it, 100)
    e_dg = gu.rel_err(dg, ds.g[f"vc_{tag}_dg"])
    e_obj = gu.rel_err(obj, ds.g[f"vc_{tag}_obj"])
    print(f"delta_G rel err {e_dg:.2e}, objective rel err {e_obj:.2e}")
    assert dg.shape[0] == it and e_dg <= 1e-9 and e_obj <= 1e-9


def test_vc_arguments():
    ds, prm = gu.load_vc("vc_c1")
    with GPLVM(ds.y, ds.z, ds.ls, prm.X, ds.M, ds.Q) as m:
        with pytest.raises(GplError):
            m.vc_fit(0, 10)
        with pytest.raises(GplError):
            m.vc_fit(1, 0)

"""The seeded synthetic generator that stands in for the benchmark's data: the same seed gives
the same bytes, the covariate design has the documented composition (the benchmark's model is
P = 236 columns with 132 dense ones at M = 128), the counts are a valid gene-major CSR with
increasing cells per gene, and the gene and cell subsets are the corresponding slices."""
import numpy as np

from gaspacho2_b200 import synth


def test_seeded_and_valid():
    a = synth.make(2, 3, N=600, G=40, M=16, Q=3)
    b = synth.make(2, 3, N=600, G=40, M=16, Q=3)
    c = synth.make(2, 4, N=600, G=40, M=16, Q=3)
    for x, y in ((a.y.i, b.y.i), (a.y.p, b.y.p), (a.y.x, b.y.x), (a.ls, b.ls), (a.X0, b.X0), (a.init.T, b.init.T)):
        assert np.array_equal(x, y)
    assert not np.array_equal(a.y.x, c.y.x) or not np.array_equal(a.y.i, c.y.i)
    y = a.y
    assert y.p[0] == 0 and y.p[-1] == y.L and np.all(np.diff(y.p) >= 0)
    assert np.all((y.i >= 0) & (y.i < y.N)) and np.all(y.x > 0)
    for j in range(y.J):
        assert np.all(np.diff(y.i[y.p[j]:y.p[j + 1]]) > 0)
    assert a.X0.shape == (600, 3) and a.init.T.shape == (16, 3) and a.ls.shape == (600,)
    assert np.all(np.isfinite(a.X0)) and np.all(a.ls > 0)


def test_benchmark_design_composition():
    """Config 2: an intercept, 4 batches, 3 numeric covariates, 100 donors and the M-column GP
    block: P = 1 + 4 + 3 + 100 + 128 = 236, of which 1 + 3 + 128 = 132 are dense."""
    ds = synth.make(2, 0, N=300, G=8, M=128, Q=10, init=False)
    p, P, nh, mc, mv, mk = ds.z.model_columns(128)
    assert P == 236
    assert int(np.sum(mc == 1)) == 132
    assert sorted(int(c) for c in ds.z.c if c > 1) == [4, 100]


def test_subsets_are_slices():
    ds = synth.make(1, 2, N=500, G=30, init=False)
    sub = synth.gene_subset(ds, 7)
    assert sub.y.J == 7 and sub.y.N == ds.y.N
    L = int(ds.y.p[7])
    assert np.array_equal(sub.y.i, ds.y.i[:L]) and np.array_equal(sub.y.x, ds.y.x[:L])
    cells = np.array([5, 0, 77, 300, 499])
    cs = synth.cell_subset(ds, cells, init=False)
    dense = np.zeros((ds.y.J, ds.y.N))
    for j in range(ds.y.J):
        dense[j, ds.y.i[ds.y.p[j]:ds.y.p[j + 1]]] = ds.y.x[ds.y.p[j]:ds.y.p[j + 1]]
    dsub = np.zeros((cs.y.J, cs.y.N))
    for j in range(cs.y.J):
        dsub[j, cs.y.i[cs.y.p[j]:cs.y.p[j + 1]]] = cs.y.x[cs.y.p[j]:cs.y.p[j + 1]]
    assert np.array_equal(dsub, dense[:, cells])
    assert np.array_equal(cs.ls, ds.ls[cells])

"""The reference driver's on-disk formats (gaspacho2_b200/formats.py): byte layouts and round
trips of the counts, the covariate design, the parameter files with and without the checkpoint
header, and the model-column map the reference loader builds from a design."""
import os

import numpy as np
import pytest

from gaspacho2_b200 import formats


def _counts(rng, N=37, J=5):
    ps, cells, vals = [0], [], []
    for _ in range(J):
        k = int(rng.integers(0, N // 2))
        cells.extend(np.sort(rng.choice(N, k, replace=False)))
        vals.extend(rng.integers(1, 9, k).astype(np.float64))
        ps.append(len(cells))
    return formats.Counts(N, J, np.array(cells, np.int32), np.array(ps, np.int32), np.array(vals))


def _design(rng, N=37):
    c = np.array([3, 1, 4], np.int32)
    v = np.array([1, 2, 1], np.int32)
    cols = [rng.integers(0, 3, N).astype(np.int32), rng.standard_normal((N, 2)), rng.integers(0, 4, N).astype(np.int32)]
    return formats.Design(N, c, v, cols)


def test_counts_layout_and_round_trip(tmp_path):
    y = _counts(np.random.default_rng(1))
    path = str(tmp_path / "Y.bin")
    formats.write_counts(path, y)
    assert os.path.getsize(path) == 4 * 3 + 4 * y.L + 4 * (y.J + 1) + 8 * y.L
    head = np.fromfile(path, np.int32, 3)
    assert list(head) == [y.N, y.J, y.L]
    back = formats.read_counts(path)
    assert (back.N, back.J) == (y.N, y.J)
    assert np.array_equal(back.i, y.i) and np.array_equal(back.p, y.p) and np.array_equal(back.x, y.x)
    with open(path, "r+b") as f:
        f.truncate(os.path.getsize(path) - 8)
    with pytest.raises(ValueError):
        formats.read_counts(path)


def test_design_layout_and_round_trip(tmp_path):
    z = _design(np.random.default_rng(2))
    path = str(tmp_path / "Z.bin")
    formats.write_design(path, z)
    # header, c, v, then the categorical codes (int32 N) and the numeric block (float64 N x 2)
    assert os.path.getsize(path) == 8 + 8 * z.n_var + 4 * z.N + 8 * z.N * 2 + 4 * z.N
    back = formats.read_design(path)
    assert np.array_equal(back.c, z.c) and np.array_equal(back.v, z.v)
    for a, b in zip(back.columns, z.columns):
        assert np.array_equal(np.asarray(a).reshape(np.asarray(b).shape), b)
    # the numeric block is stored column-major
    raw = np.fromfile(path, np.float64, offset=8 + 8 * z.n_var + 4 * z.N, count=2 * z.N)
    assert np.array_equal(raw, z.columns[1].ravel(order="F"))


def test_model_columns_and_matrix():
    z = _design(np.random.default_rng(3))
    M = 6
    p, P, nh, mc, mv, mk = z.model_columns(M)
    # intercept, the three file variables (3 levels, 2 numeric columns, 4 levels), the GP block
    assert p == 5 and P == 1 + 3 + 2 + 4 + M
    assert list(nh) == [0, 1, 4, 6, 10, 10 + M]
    assert list(mk[:10]) == [0, 1, 1, 1, 2, 2, 3, 3, 3, 3]
    Knm = np.random.default_rng(4).standard_normal((z.N, M))
    Zm = z.dense_model_matrix(M, Knm)
    assert np.all(Zm[:, 0] == 1.0)
    assert np.all(Zm[:, 1:4].sum(axis=1) == 1.0) and np.all(Zm[:, 6:10].sum(axis=1) == 1.0)
    assert np.array_equal(np.argmax(Zm[:, 1:4], axis=1), z.columns[0])
    assert np.array_equal(Zm[:, 4:6], z.columns[1]) and np.array_equal(Zm[:, 10:], Knm)


@pytest.mark.parametrize("header", [False, True])
def test_params_round_trip(tmp_path, header):
    rng = np.random.default_rng(5)
    N, J, M, p, Q = 11, 4, 3, 5, 2
    prm = formats.Params(rng.random(N), rng.random(p), rng.standard_normal((N, Q)), rng.standard_normal((M, Q)),
                         rng.random(Q), rng.random(J))
    path = str(tmp_path / "params.bin")
    formats.write_params(path, prm, header=(N, J, M, 17, p, Q) if header else None)
    n_doubles = N + p + N * Q + M * Q + Q + J
    assert os.path.getsize(path) == (24 if header else 0) + 8 * n_doubles
    back = formats.read_params(path, 0, 0, 0, 0, 0, header=True) if header else formats.read_params(path, N, J, M, p, Q)
    for a, b in zip(back.flat(), prm.flat()):
        assert np.array_equal(a, b)
    # X is stored column-major: the first N doubles after Omega and delta are X[:, 0]
    flat = np.fromfile(path, np.float64, offset=24 if header else 0)
    assert np.array_equal(flat[N + p:N + p + N], prm.X[:, 0])
    with pytest.raises(ValueError):
        formats.read_params(path, N + 1, J, M, p, Q, header=False) if not header else formats.read_params(
            path, N, J + 100, M, p, Q, header=False)


def test_doubles_length_checked(tmp_path):
    path = str(tmp_path / "ls.bin")
    formats.write_doubles(path, np.arange(7.0))
    assert np.array_equal(formats.read_doubles(path, 7), np.arange(7.0))
    with pytest.raises(ValueError):
        formats.read_doubles(path, 8)

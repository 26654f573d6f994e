"""The ggplvm CLI: the reference driver's command line, input formats and output files.

CPU tests cover argument and input-file errors (answered before any device work); the GPU
test runs a budgeted fit of the c0_small fixture through the CLI and compares params.bin,
Params9.bin, beta.bin, X9.gz and phi.gz with the reference's own fit of the same inputs
(ggplvm.cu:1301-1346 for the file layouts), plus the genotype score statistics of the
differential-expression driver (ScoreStats.gz, ggplvm_de.cu:1205-1214)."""
import gzip
import os
import subprocess

import numpy as np
import pytest

from gaspacho2_b200 import build as gbuild
from gaspacho2_b200 import formats
from tests import golden_util as gu

TOL_FIT = 1e-6


@pytest.fixture(scope="module")
def cli():
    gbuild.build()
    assert os.path.exists(gbuild.CLI), "CLI was not built"
    return gbuild.CLI


def _inputs(tmp_path, gd):
    paths = formats.write_dataset(str(tmp_path), gd.y, gd.z, gd.ls, gd.X0, init=gd.init)
    return paths


def _run(cli, args, cwd):
    return subprocess.run([cli] + [str(a) for a in args], cwd=cwd, capture_output=True, text=True, timeout=600)


def test_usage_errors(cli, tmp_path):
    r = _run(cli, [], tmp_path)
    assert r.returncode == 2 and "usage" in r.stderr
    r = _run(cli, ["a", "b", "c", "d", "--precision", "fp16"], tmp_path)
    assert r.returncode == 2
    r = _run(cli, ["a", "b", "c", "d", "-M", "x"], tmp_path)
    assert r.returncode == 2
    r = _run(cli, ["a", "b", "c", "d", "--bogus"], tmp_path)
    assert r.returncode == 2


def test_input_errors_before_device_work(cli, tmp_path):
    gd = gu.load("c0_small")
    p = _inputs(tmp_path, gd)
    r = _run(cli, [tmp_path / "absent.bin", p["Z"], p["ls"], p["Xi"], "-M", gd.M, "-Q", gd.Q], tmp_path)
    assert r.returncode == 1 and "cannot open" in r.stderr
    trunc = tmp_path / "Ytrunc.bin"
    trunc.write_bytes(open(p["Y"], "rb").read()[:-8])
    r = _run(cli, [trunc, p["Z"], p["ls"], p["Xi"], "-M", gd.M, "-Q", gd.Q], tmp_path)
    assert r.returncode == 1 and "truncated" in r.stderr
    short_ls = tmp_path / "ls_short.bin"
    np.zeros(gd.N - 1).tofile(short_ls)
    r = _run(cli, [p["Y"], p["Z"], short_ls, p["Xi"], "-M", gd.M, "-Q", gd.Q], tmp_path)
    assert r.returncode == 1 and "truncated" in r.stderr


def _read_gz_rows(path):
    with gzip.open(path, "rt") as f:
        return [line.rstrip("\n") for line in f]


@pytest.mark.gpu
def test_cli_fit_matches_reference_fit(cli, tmp_path):
    gd = gu.load("c0_small")
    p = _inputs(tmp_path, gd)
    out = tmp_path / "out"
    out.mkdir()
    budget = 12
    G = gd.g["score_G"]
    G.T.tofile(tmp_path / "G.bin")  # column-major N x L
    r = _run(cli, [p["Y"], p["Z"], p["ls"], p["Xi"], "-M", gd.M, "-Q", gd.Q, "--init-params", p["params"],
                   "--max-outer", 1, "--max-lbfgs-iters", budget, "--out-dir", out, "--quiet",
                   "--genotypes", tmp_path / "G.bin", "-L", G.shape[1]], tmp_path)
    assert r.returncode == 0, r.stderr
    N, J, M, Q = gd.N, gd.J, gd.M, gd.Q
    p_ = gd.init.delta.shape[0]
    g = gd.g
    prm = formats.read_params(str(out / "params.bin"), N, J, M, p_, Q)
    for name, a in (("Omega", prm.Omega), ("delta", prm.delta), ("X", prm.X.T.ravel()), ("T", prm.T.T.ravel()),
                    ("rho", prm.rho), ("phi", prm.phi)):
        err = gu.rel_err(a, g["fit_" + name])
        assert err <= TOL_FIT, (name, err)
    P = int(g["fit_Beta"].shape[0] // J)
    beta = np.fromfile(out / "beta.bin", np.float64)
    assert beta.shape[0] == P * J
    assert gu.rel_err(beta, g["fit_Beta"]) <= TOL_FIT
    # Params9.bin: header then the same blocks as params.bin
    hdr = np.fromfile(out / "Params9.bin", np.int32, 6)
    assert list(hdr) == [N, J, M, P, p_, Q]
    p9 = formats.read_params(str(out / "Params9.bin"), N, J, M, p_, Q, header=True)
    assert np.array_equal(p9.X, prm.X) and np.array_equal(p9.phi, prm.phi)
    # X9.gz: N rows of X, M rows of T, one row of rho, "%lf," per value
    rows = _read_gz_rows(out / "X9.gz")
    assert len(rows) == N + M + 1
    first = [float(s) for s in rows[0].split(",") if s]
    assert len(first) == Q and np.allclose(first, prm.X[0], atol=5e-7)
    assert rows[0] == "".join("%f," % v for v in prm.X[0])
    # phi.gz: the reference writes the first J values of its Omega buffer
    phi_rows = _read_gz_rows(out / "phi.gz")
    assert len(phi_rows) == J
    assert phi_rows[:3] == ["%f" % v for v in prm.Omega[:3]]
    # ScoreStats.gz: J rows of L "%lf," values, the same statistics as the C ABI at the fitted state
    srows = _read_gz_rows(out / "ScoreStats.gz")
    assert len(srows) == J
    S_cli = np.array([[float(v) for v in row.split(",") if v] for row in srows])
    assert S_cli.shape == (J, G.shape[1]) and np.all(np.isfinite(S_cli))
    from gaspacho2_b200 import GPLVM
    with GPLVM.from_dataset(gd) as m:
        m.set_params(gd.init)
        m.kernel_mats()
        m.glm_init()
        m.fit(1, budget)
        S_api = m.score_stats(G)
    assert np.allclose(S_cli, S_api, rtol=0, atol=1e-6)
    tau = np.fromfile(out / "Tau.bin", np.float64)
    assert tau.shape[0] == M * Q
    assert np.allclose(tau[:M], (np.arange(1, M + 1) / (M + 1)) * 2.0 * 3.14159265358979, rtol=0, atol=1e-15)

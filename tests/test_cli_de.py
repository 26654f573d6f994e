"""The ggplvm_de CLI: the reference DE driver's command line (ggplvm_de.cu:886-1237) and its
output files. CPU tests cover usage and input errors (answered before any device work); the
GPU test runs the model comparison of the de_c1 fixture with 3 sweeps per model and compares
BFs_de.gz with the reference's table, and the appended Beta_de.gz / Knm_de.gz with the C ABI's
view of the same models."""
import gzip
import os
import subprocess

import numpy as np
import pytest

from gaspacho2_b200 import build as gbuild
from gaspacho2_b200 import formats
from tests import golden_util as gu


@pytest.fixture(scope="module")
def cli():
    gbuild.build()
    exe = os.path.join(gbuild.PKG, "bin", "ggplvm_de")
    assert os.path.exists(exe), "ggplvm_de was not built"
    return exe


def _run(cli, args, cwd):
    return subprocess.run([cli] + [str(a) for a in args], cwd=cwd, capture_output=True, text=True, timeout=600)


def _rows(path):
    with gzip.open(path, "rt") as f:
        return [np.array([float(v) for v in line.rstrip(",\n").split(",")]) for line in f]


def test_usage_errors(cli, tmp_path):
    r = _run(cli, [], tmp_path)
    assert r.returncode == 2 and "usage" in r.stderr
    r = _run(cli, ["a", "b", "c"], tmp_path)  # no --init-params
    assert r.returncode == 2 and "--init-params" in r.stderr
    r = _run(cli, ["a", "b", "c", "--init-params", "p", "-L", "2"], tmp_path)  # G.bin and dox.bin missing
    assert r.returncode == 2
    r = _run(cli, ["a", "b", "c", "--init-params", "p", "-Mf", "0"], tmp_path)
    assert r.returncode == 2


def test_input_errors_before_device_work(cli, tmp_path):
    gd = gu.load("de_c1")
    p = formats.write_dataset(str(tmp_path), gd.y, gd.z, gd.ls, gd.X0, init=gd.init)
    r = _run(cli, [tmp_path / "absent.bin", p["Z"], p["ls"], "--init-params", p["params"], "-Mf", gd.M, "-Q", gd.Q],
             tmp_path)
    assert r.returncode == 1 and "cannot open" in r.stderr
    short = tmp_path / "params_short.bin"
    short.write_bytes(open(p["params"], "rb").read()[:-16])
    r = _run(cli, [p["Y"], p["Z"], p["ls"], "--init-params", short, "-Mf", gd.M, "-Q", gd.Q], tmp_path)
    assert r.returncode == 1 and "truncated" in r.stderr


@pytest.mark.gpu
def test_cli_de_matches_reference(cli, tmp_path):
    gd = gu.load("de_c1")
    p = formats.write_dataset(str(tmp_path), gd.y, gd.z, gd.ls, gd.X0, init=gd.init)
    out = tmp_path / "out"
    out.mkdir()
    Mr = int(gd.g["in_Mredc"])
    r = _run(cli, [p["Y"], p["Z"], p["ls"], "--init-params", p["params"], "-Mf", gd.M, "-Mr", Mr, "-Q", gd.Q,
                   "--max-sweeps", 3, "--out-dir", out, "--quiet"], tmp_path)
    assert r.returncode == 0, r.stderr
    bfs = np.array(_rows(out / "BFs_de.gz"))
    ref = gd.g["de_j3_BFs"]
    assert bfs.shape == ref.shape
    assert np.allclose(bfs, ref, rtol=1e-8, atol=1.5e-6)  # "%lf" keeps 6 decimals
    beta = _rows(out / "Beta_de.gz")
    assert len(beta) == gd.J * (gd.Q + 1)  # J rows per GP model
    assert np.allclose(np.array(beta[-gd.J:]).T, gd.g["de_j3_beta_full"], rtol=1e-6, atol=1e-5)
    knm = _rows(out / "Knm_de.gz")
    assert len(knm) == gd.Q * (gd.N + Mr) + gd.N + gd.M


# ---- ggplvm_delta: the variance-component driver's command line (ggplvm_delta.cu:784-1097) ----
@pytest.fixture(scope="module")
def cli_vc():
    gbuild.build()
    exe = os.path.join(gbuild.PKG, "bin", "ggplvm_delta")
    assert os.path.exists(exe), "ggplvm_delta was not built"
    return exe


def test_vc_usage_errors(cli_vc, tmp_path):
    r = _run(cli_vc, [], tmp_path)
    assert r.returncode == 2 and "usage" in r.stderr
    r = _run(cli_vc, ["a", "b", "c", "d", "--init-deltaG", "-1"], tmp_path)
    assert r.returncode == 2
    r = _run(cli_vc, ["a", "b", "c", "d", "--bogus"], tmp_path)
    assert r.returncode == 2


def _vc_inputs(tmp_path):
    ds, prm = gu.load_vc("vc_c1")
    p = formats.write_dataset(str(tmp_path), ds.y, ds.z, ds.ls, ds.X0)
    # params.bin as the driver reads it: Omega, the fit's p - 1 deltas, X, T, rho (and phi)
    with open(tmp_path / "params.bin", "wb") as f:
        for a in (prm.Omega, prm.delta, prm.X.ravel(order="F"), prm.T.ravel(order="F"), prm.rho, prm.phi):
            np.asarray(a, np.float64).tofile(f)
    return ds, p


def test_vc_missing_params_file(cli_vc, tmp_path):
    ds, p = _vc_inputs(tmp_path)
    os.remove(tmp_path / "params.bin")
    r = _run(cli_vc, [p["Y"], p["Z"], p["ls"], p["Xi"], "-M", ds.M, "-Q", ds.Q], tmp_path)
    assert r.returncode == 1 and "cannot open" in r.stderr


@pytest.mark.gpu
def test_cli_vc_matches_reference(cli_vc, tmp_path):
    ds, p = _vc_inputs(tmp_path)
    r = _run(cli_vc, [p["Y"], p["Z"], p["ls"], p["Xi"], "-M", ds.M, "-Q", ds.Q, "--max-outer", 3, "--quiet"],
             tmp_path)
    assert r.returncode == 0, r.stderr
    rows = [line.split() for line in r.stdout.splitlines() if line.startswith("itr=")]
    dg = np.array([float(x[1].split("=")[1]) for x in rows])
    obj = np.array([float(x[2].split("=")[1]) for x in rows])
    assert np.allclose(dg, ds.g["vc_i3_dg"], rtol=1e-9, atol=0)
    assert np.allclose(obj, ds.g["vc_i3_obj"], rtol=1e-9, atol=0)

"""CPU replay of the memory indexing of the batched Cholesky and inverse panel kernels, and of the
linear predictor and the W / nu pass.

tests/index_mirror/k_inv_mirror.c mirrors every shared- and global-memory index of
k_potrf_panel, k_trtri_panel and k_lauum_panel (gaspacho2_b200/csrc/k_inv.cu) and counts the
outputs each must write. It runs here for every P from 1 up to the largest P the launchers
admit (read from k_inv.cu), so no size the GPU path can reach goes unchecked; one P past the
Cholesky panel's limit shows that the mirror does catch the rows its update would leave out.

tests/index_mirror/k_wnu_eta_mirror.c mirrors k_eta_dmma (both tile heights), k_level_sums,
k_w_nu, k_w_nu_counts, k_zt_u (its three modes), k_hk and k_group_sums_dmma over a sweep of cell, gene, dense-column,
group and cell-range counts (odd sizes, ragged slices, persistent grids that stride, empty
ranges) and counts every output and every loaded cell; with the level sums' rows planted
unpadded, or Z^T u's cell ranges planted at odd starts, it must fail.
"""
import os
import re
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "index_mirror", "k_inv_mirror.c")
KINV = os.path.join(os.path.dirname(HERE), "gaspacho2_b200", "csrc", "k_inv.cu")


def _limit(name):
    m = re.search(rf"constexpr int {name} = (\d+);", open(KINV).read())
    assert m, f"{name} not found in k_inv.cu"
    return int(m.group(1))


@pytest.fixture(scope="module")
def mirror(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("mirror") / "k_inv_mirror")
    subprocess.run(["gcc", "-O2", "-std=c11", "-o", exe, SRC], check=True)
    return exe


@pytest.mark.parametrize("kernel,limit", [("potrf", "kPotrfMaxP"), ("trtri", "kInverseMaxP"),
                                          ("lauum", "kInverseMaxP")])
def test_every_admitted_size_stays_in_bounds(mirror, kernel, limit):
    top = _limit(limit)
    r = subprocess.run([mirror, kernel, "1", str(top)], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    assert r.stdout.strip() == f"ok {kernel} 1..{top}"


def test_inverse_limit_is_the_shared_memory_limit():
    """kInverseMaxP is the largest P whose panel fits the launcher's 220 KiB."""
    ib, is_, ls = 32, 36, 33

    def smem(P):
        nb = (P + ib - 1) // ib
        return 8 * (nb * ib * is_ + 2 * ib * is_ + 2 * ib * ls + ib)

    top = _limit("kInverseMaxP")
    assert smem(top) <= 220 * 1024 < smem(top + 1)


def test_mirror_flags_rows_the_cholesky_update_misses(mirror):
    top = _limit("kPotrfMaxP")
    r = subprocess.run([mirror, "potrf", str(top + 1), str(top + 1)], capture_output=True, text=True)
    assert r.returncode == 1
    assert "updated 0 times" in r.stderr


@pytest.fixture(scope="module")
def wnu_mirror(tmp_path_factory):
    exe = str(tmp_path_factory.mktemp("mirror") / "k_wnu_eta_mirror")
    subprocess.run(["gcc", "-O2", "-std=c11", "-o", exe, os.path.join(HERE, "index_mirror", "k_wnu_eta_mirror.c")],
                   check=True)
    return exe


def test_predictor_and_w_nu_stay_in_bounds(wnu_mirror):
    r = subprocess.run([wnu_mirror], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr[-2000:]
    lines = r.stdout.split()
    for name in ("eta4", "eta2", "levels", "w_nu", "counts", "zt_u", "hk", "group_sums"):
        assert name in lines, r.stdout


def test_mirror_flags_unpadded_level_sums(wnu_mirror):
    r = subprocess.run([wnu_mirror, "plant"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 1
    assert "level sum alignment" in r.stderr


def test_mirror_flags_odd_cell_ranges(wnu_mirror):
    r = subprocess.run([wnu_mirror, "plant-odd"], capture_output=True, text=True, timeout=600)
    assert r.returncode == 1
    assert "alignment" in r.stderr or "odd range start" in r.stderr

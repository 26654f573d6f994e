"""Seeded synthetic single-cell count data for the GP-LVM fit, with the reference's file layouts.

The reference publishes no dataset, so every workload is synthetic. ``make(config, seed)``
builds one of the configurations below:

==========  =========  ========  =====  ====  =========================================
config      N cells    G genes   M      Q     covariates (file variables)
==========  =========  ========  =====  ====  =========================================
0           2,000      500       32     2     batch (2 levels), 1 numeric
1           20,000     2,000     64     5     batch (4 levels), 3 numerics
2           100,000    10,000    128    10    batch (4), 3 numerics, donor (100 levels)
4           500,000    5,000     256    10    batch (4), 3 numerics, donor (300 levels)
==========  =========  ========  =====  ====  =========================================

Generative model (per gene g, cell n):
``log rate = mu_g + f_g(x_n) + log s_n + c_n . beta_g (+ donor effect)``, counts Poisson.
``x_n ~ N(0, I_Q)``; ``s_n ~ LogNormal(0, 0.3^2)``; numerics ``N(0, 1)``; covariate
effects ``N(0, 0.2^2)``; donor effects ``N(0, 0.3^2)``; ``mu_g ~ N(mu0, sd^2)`` per config.
``f_g`` is an ARD-RBF GP draw (variance 1, lengthscale 1) realised with 256 random Fourier
features, which keeps a 100K-cell draw linear in N. The stated mu distributions together
with the GP and covariate terms give fewer zeros than the stated targets (about 85% at
config 0, 90% at config 1, 92% at config 4), so those configs shift every mu_g by a
constant (``shift``) calibrated to the target; config 2 states no target and is unshifted.

Initialisation (not part of the reference, which reads it from files): ``X0`` = top-Q PCA
scores of ``log1p(y / s)`` scaled to unit variance; ``T0`` = k-means centres of ``X0``;
the other parameters take the reference defaults (init.cu:27-48).
"""
from __future__ import annotations

import dataclasses
from concurrent.futures import ThreadPoolExecutor
from typing import Optional

import numpy as np

from .formats import Counts, Design, Params

CONFIGS = {
    0: dict(N=2000, G=500, M=32, Q=2, batch=2, n_num=1, donors=0, mu=(-1.0, 1.0), shift=-1.6),
    1: dict(N=20000, G=2000, M=64, Q=5, batch=4, n_num=3, donors=0, mu=(-1.5, 1.2), shift=-1.75),
    2: dict(N=100000, G=10000, M=128, Q=10, batch=4, n_num=3, donors=100, mu=(-2.0, 1.5), shift=0.0),
    4: dict(N=500000, G=5000, M=256, Q=10, batch=4, n_num=3, donors=300, mu=(-2.0, 1.5), shift=-0.8,
            variants=20, interaction_frac=0.05),
}

N_RFF = 256


@dataclasses.dataclass
class Dataset:
    config: dict
    seed: int
    y: Counts
    z: Design
    ls: np.ndarray
    X0: np.ndarray
    init: Params
    M: int
    Q: int
    X_true: np.ndarray
    # genotypes (configurations with cis variants): donor dosages [donors][genes][variants] in
    # {0, 1, 2} and the truth of their effects (causal variant, main effect, interaction effect)
    genotypes: Optional[np.ndarray] = None
    geno_truth: Optional[dict] = None

    @property
    def N(self) -> int:
        return self.y.N

    @property
    def J(self) -> int:
        return self.y.J

    def zero_fraction(self) -> float:
        return 1.0 - self.y.L / float(self.y.N) / float(self.y.J)


def default_params(N: int, J: int, p: int, M: int, Q: int, X0: np.ndarray, T0: np.ndarray) -> Params:
    """The reference defaults (initParams, init.cu:27-48) around given X and T."""
    delta = np.full(p, 0.01)
    delta[0] = 1.5
    delta[p - 1] = 0.3
    rho = np.full(Q, 10.0)
    rho[0] = 5.0
    return Params(np.ones(N), delta, np.asarray(X0, np.float64), np.asarray(T0, np.float64), rho, np.ones(J))


def _kmeans(X: np.ndarray, k: int, rng: np.random.Generator, iters: int = 25) -> np.ndarray:
    n = X.shape[0]
    C = X[rng.choice(n, size=k, replace=False)].copy()
    for _ in range(iters):
        d = (X * X).sum(1)[:, None] - 2.0 * X @ C.T + (C * C).sum(1)[None, :]
        lab = d.argmin(1)
        for m in range(k):
            sel = lab == m
            if sel.any():
                C[m] = X[sel].mean(0)
    return C


def _pca_scores(y: Counts, ls: np.ndarray, Q: int, seed: int) -> np.ndarray:
    """Top-Q principal component scores of log1p(y / s), centred per gene, unit variance."""
    import scipy.sparse as sp
    import scipy.sparse.linalg as spla

    N, J = y.N, y.J
    gene = np.repeat(np.arange(J, dtype=np.int64), np.diff(y.p))
    vals = np.log1p(y.x / ls[y.i])
    A = sp.csr_matrix((vals, (y.i.astype(np.int64), gene)), shape=(N, J))
    mean = np.asarray(A.mean(axis=0)).ravel()
    if N * J <= 4_000_000:
        D = A.toarray() - mean[None, :]
        U, S, _ = np.linalg.svd(D, full_matrices=False)
        scores = U[:, :Q] * S[:Q]
    else:
        op = spla.LinearOperator(
            (N, J), dtype=np.float64,
            matvec=lambda v: A @ v - (mean @ v) * np.ones(N),
            rmatvec=lambda u: A.T @ u - mean * u.sum(),
        )
        v0 = np.random.default_rng(seed).standard_normal(min(N, J))
        U, S, _ = spla.svds(op, k=Q, v0=v0, random_state=seed)
        order = np.argsort(-S)
        scores = U[:, order] * S[order]
    scores = scores - scores.mean(0)
    sd = scores.std(0)
    sd[sd == 0] = 1.0
    return scores / sd


def make(config: int = 0, seed: int = 0, N: Optional[int] = None, G: Optional[int] = None,
         M: Optional[int] = None, Q: Optional[int] = None, init: bool = True, threads: int = 8) -> Dataset:
    """Builds a seeded dataset for ``config``; N, G, M, Q override the table for small cases."""
    cfg = dict(CONFIGS[config])
    for k, val in (("N", N), ("G", G), ("M", M), ("Q", Q)):
        if val is not None:
            cfg[k] = int(val)
    N, G, M, Q = cfg["N"], cfg["G"], cfg["M"], cfg["Q"]
    ss = np.random.SeedSequence([seed, config])
    rng = np.random.default_rng(ss.spawn(1)[0])

    X = rng.standard_normal((N, Q))
    s = np.exp(rng.normal(0.0, 0.3, N))
    batch = rng.integers(0, cfg["batch"], N).astype(np.int32)
    num = rng.standard_normal((N, cfg["n_num"]))
    donors = cfg["donors"]
    donor = rng.integers(0, donors, N).astype(np.int32) if donors else None
    mu = rng.normal(cfg["mu"][0], cfg["mu"][1], G) + cfg["shift"]
    b_batch = rng.normal(0.0, 0.2, (cfg["batch"], G))
    b_num = rng.normal(0.0, 0.2, (cfg["n_num"], G))
    d_eff = rng.normal(0.0, 0.3, (donors, G)) if donors else None
    W_rff = rng.standard_normal((Q, N_RFF))
    b_rff = rng.uniform(0.0, 2.0 * np.pi, N_RFF)
    A_rff = rng.standard_normal((N_RFF, G))
    Phi = np.sqrt(2.0 / N_RFF) * np.cos(X @ W_rff + b_rff)
    base = np.log(s) + 0.0

    chunk = max(1, min(G, 2_000_000 // max(N, 1)))
    starts = list(range(0, G, chunk))
    child = ss.spawn(len(starts) + 1)[1:]

    # cis genotypes (configurations with `variants`): per gene, that many variants with allele
    # frequencies U(0.05, 0.5) and donor dosages Binomial(2, p); one causal variant per gene adds a
    # main effect N(0, 0.1^2) to the log-rate, and on a fraction of genes also an interaction
    # N(0, 0.1^2) x dosage x f_g(x) with the gene's GP draw f_g
    V = int(cfg.get("variants", 0))
    geno = truth = None
    if V and donors:
        grng = np.random.default_rng(ss.spawn(5)[4])
        freq = grng.uniform(0.05, 0.5, (G, V))
        geno = grng.binomial(2, freq[None, :, :], (donors, G, V)).astype(np.int8)
        causal = grng.integers(0, V, G)
        main = grng.normal(0.0, 0.1, G)
        inter = np.where(grng.random(G) < cfg.get("interaction_frac", 0.0), grng.normal(0.0, 0.1, G), 0.0)
        dos_c = geno[:, np.arange(G), causal].astype(np.float64)  # donors x genes, the causal dosage
        truth = {"causal": causal, "main": main, "interaction": inter, "freq": freq}

    def gen(ci: int):
        g0 = starts[ci]
        g1 = min(G, g0 + chunk)
        crng = np.random.default_rng(child[ci])
        f = Phi @ A_rff[:, g0:g1]
        lr = f.copy()
        lr += mu[g0:g1][None, :] + base[:, None]
        lr += b_batch[batch, g0:g1] + num @ b_num[:, g0:g1]
        if donors:
            lr += d_eff[donor, g0:g1]
        if geno is not None:
            dc = dos_c[donor, g0:g1]
            lr += dc * main[None, g0:g1] + dc * inter[None, g0:g1] * f
        cnt = crng.poisson(np.exp(lr))
        gi, ci_ = np.nonzero(cnt.T)  # gene-major, cells ascending within a gene
        return g1 - g0, gi, ci_.astype(np.int32), cnt.T[gi, ci_].astype(np.float64)

    with ThreadPoolExecutor(max_workers=threads) as ex:
        parts = list(ex.map(gen, range(len(starts))))
    nnz_per_gene = []
    cells, vals = [], []
    for ng, gi, ci_, xv in parts:
        nnz_per_gene.append(np.bincount(gi, minlength=ng))
        cells.append(ci_)
        vals.append(xv)
    p = np.zeros(G + 1, np.int64)
    p[1:] = np.cumsum(np.concatenate(nnz_per_gene))
    if p[-1] >= 2 ** 31:
        raise ValueError("more than 2^31-1 nonzeros: the reference CSR uses int32 offsets")
    y = Counts(N, G, np.concatenate(cells).astype(np.int32), p.astype(np.int32), np.concatenate(vals))

    c = [cfg["batch"]] + [1] * cfg["n_num"] + ([donors] if donors else [])
    v = [1] * len(c)
    cols = [batch] + [num[:, k:k + 1].copy() for k in range(cfg["n_num"])] + ([donor] if donors else [])
    z = Design(N, np.array(c, np.int32), np.array(v, np.int32), cols)

    p_vars = len(c) + 2
    if init:
        X0 = _pca_scores(y, s, Q, seed)
        T0 = _kmeans(X0, M, np.random.default_rng(ss.spawn(3)[2]))
    else:
        X0 = X.copy()
        T0 = _kmeans(X0, M, np.random.default_rng(ss.spawn(3)[2]), iters=5)
    prm = default_params(N, G, p_vars, M, Q, X0, T0)
    return Dataset(cfg, seed, y, z, s, X0, prm, M, Q, X, geno, truth)


def cell_subset(ds: Dataset, cells: np.ndarray, init: bool = True) -> Dataset:
    """The cells ``cells`` of ``ds`` (in that order) with every gene: the counts, covariates, size
    factors and true coordinates of those cells, drawn from the same gene parameters. With
    ``init`` the start is computed on the subset as ``make`` computes it (PCA of log1p, k-means)."""
    cells = np.asarray(cells, np.int64)
    y = ds.y
    new = np.full(y.N, -1, np.int64)
    new[cells] = np.arange(cells.shape[0])
    gene = np.repeat(np.arange(y.J), np.diff(np.asarray(y.p, np.int64)))
    keep = new[y.i] >= 0
    ni, ng, nx = new[y.i][keep], gene[keep], y.x[keep]
    o = np.lexsort((ni, ng))  # gene-major, cells ascending within a gene
    p = np.zeros(y.J + 1, np.int64)
    p[1:] = np.cumsum(np.bincount(ng, minlength=y.J))
    ys = Counts(int(cells.shape[0]), y.J, ni[o].astype(np.int32), p.astype(np.int32), nx[o].copy())
    cols = [np.asarray(col)[cells].copy() for col in ds.z.columns]
    z = Design(int(cells.shape[0]), ds.z.c.copy(), ds.z.v.copy(), cols)
    s = np.asarray(ds.ls)[cells].copy()
    Xt = np.asarray(ds.X_true)[cells].copy()
    if init:
        X0 = _pca_scores(ys, s, ds.Q, ds.seed)
        T0 = _kmeans(X0, ds.M, np.random.default_rng([ds.seed, 7]))
    else:
        X0 = np.asarray(ds.X0)[cells].copy()
        T0 = np.asarray(ds.init.T).copy()
    prm = default_params(ys.N, ys.J, len(ds.z.c) + 2, ds.M, ds.Q, X0, T0)
    return Dataset(ds.config, ds.seed, ys, z, s, X0, prm, ds.M, ds.Q, Xt)


def gene_subset(ds: Dataset, n_genes: int) -> Dataset:
    """The first ``n_genes`` genes of ``ds`` (cells and covariates unchanged)."""
    y = ds.y
    n_genes = min(n_genes, y.J)
    L = int(y.p[n_genes])
    ys = Counts(y.N, n_genes, y.i[:L].copy(), y.p[:n_genes + 1].copy(), y.x[:L].copy())
    init = dataclasses.replace(ds.init, phi=ds.init.phi[:n_genes].copy())
    return dataclasses.replace(ds, y=ys, init=init)

"""Generates the golden vectors in tests/golden/ from the reference's own kernels.

The reference publishes no test vectors, so these fixtures are produced by running the
reference source itself (compiled for the host by ``make -C oracle ref`` from the
reference checkout) on small seeded inputs, phase by phase in the reference driver's
order (ggplvm.cu:1101-1330). Each fixture stores its inputs too, so tests do not depend
on the generator's random streams. Run from the repository root:

    make -C oracle ref && python tests/golden/make_golden.py
"""
from __future__ import annotations

import os
import sys

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, ROOT)

from gaspacho2_b200 import synth  # noqa: E402
from gaspacho2_b200.formats import Counts  # noqa: E402
from oracle import refcpu  # noqa: E402

OUT = os.path.dirname(os.path.abspath(__file__))


def edge_counts(ds):
    """Adds the count-handling edge cases the reference's merge walk defines
    (ggplvm.cu:505-511): an all-zero gene, a gene with every cell nonzero, a gene whose
    entries go out of order (the walk stops at the first non-increasing index) and a
    gene with a duplicated index."""
    y = ds.y
    N = y.N
    genes_i = [y.i[y.p[j]:y.p[j + 1]] for j in range(y.J)]
    genes_x = [y.x[y.p[j]:y.p[j + 1]] for j in range(y.J)]
    genes_i[0] = np.zeros(0, np.int32)
    genes_x[0] = np.zeros(0)
    genes_i[1] = np.arange(N, dtype=np.int32)
    genes_x[1] = (np.arange(N) % 5 + 1).astype(np.float64)
    sizes = [g.shape[0] for g in genes_i]
    swap_gene = next(j for j in range(2, y.J) if sizes[j] >= 6)
    dup_gene = next(j for j in range(swap_gene + 1, y.J) if sizes[j] >= 4)
    gi = genes_i[swap_gene].copy()
    gi[3], gi[4] = gi[4], gi[3]
    genes_i[swap_gene] = gi
    gi = genes_i[dup_gene].copy()
    gi[2] = gi[1]
    genes_i[dup_gene] = gi
    ds.edge_genes = (swap_gene, dup_gene)
    p = np.zeros(y.J + 1, np.int64)
    p[1:] = np.cumsum([g.shape[0] for g in genes_i])
    ds.y = Counts(N, y.J, np.concatenate(genes_i).astype(np.int32), p.astype(np.int32), np.concatenate(genes_x))
    return ds


CASES = {
    "c0_small": dict(config=0, seed=1, N=300, G=40, M=8, Q=2),
    "c2_cats": dict(config=2, seed=2, N=400, G=30, M=10, Q=3),
    "edges": dict(config=1, seed=3, N=250, G=24, M=6, Q=2),
}


def make_case(name: str, spec: dict) -> dict:
    kw = dict(spec)
    cfg = kw.pop("config")
    seed = kw.pop("seed")
    ds = synth.make(cfg, seed, **kw)
    if name == "c2_cats":
        # leave one donor level without cells (an all-zero column of the model matrix)
        donor = ds.z.columns[-1]
        donor[donor == 3] = 4
    if name == "edges":
        ds = edge_counts(ds)
    m = refcpu.RefModel.from_dataset(ds)
    extra = {"edge_genes": np.array(ds.edge_genes)} if name == "edges" else {}
    out = {
        "in_N": np.array(ds.y.N), "in_J": np.array(ds.y.J), "in_M": np.array(ds.M), "in_Q": np.array(ds.Q),
        "in_y_i": ds.y.i, "in_y_p": ds.y.p, "in_y_x": ds.y.x, "in_z_c": ds.z.c, "in_z_v": ds.z.v,
        "in_z_body": np.frombuffer(ds.z.body_bytes(), np.uint8), "in_ls": ds.ls, "in_X0": ds.X0,
    }
    for k, a in zip(("Omega", "delta", "X", "T", "rho", "phi"), ds.init.flat()):
        out["in_init_" + k] = a
    m.set_params(ds.init)
    m.kernel_mats()
    for k in ("Knm", "Kmm", "Kinv", "KinvKmn", "titsias"):
        out["kmats_" + k] = m.get(k)
    m.glm_init()
    out["init_Beta"] = m.get("Beta")
    out["sweep0_lkhd"] = np.array(m.irls_sweep(0, 0))
    P = m.P
    out["sweep0_Psi3"] = m.get("Psi")[:3 * P * P]
    for k in ("Beta", "phi", "lkhds"):
        out["sweep0_" + k] = m.get(k)
    out["sweep0_W"] = m.get("W")[: m.N * m.J]
    out["sweep0_Nu"] = m.get("Nu")
    n = m.irls(0, 200)
    out["irls_n"] = np.array(n)
    out["irls_lkhd"] = m.get("lkhd")[:n]
    for k in ("Beta", "phi"):
        out["irls_" + k] = m.get(k)
    # genotype score statistics at the IRLS state (getScoreStats, ggplvm_de.cu:489-535):
    # seeded dosages 0/1/2 with allele frequencies in U(0.05, 0.5)
    rs = np.random.default_rng(1000 + spec["seed"])
    freq = rs.uniform(0.05, 0.5, size=5)
    out["score_G"] = rs.binomial(2, freq, size=(ds.y.N, 5)).astype(np.float64)
    out["score_S"] = m.score_stats(out["score_G"])
    out["obj0"] = np.array(m.objective_after_irls(0))
    out["obj0_lkhds"] = m.get("lkhds")
    out["grad0"] = m.gradient()
    for k in ("tBeta", "C1", "C2"):
        out["grad0_" + k] = m.get(k)
    m.lbfgs_update(0, 0)
    out["obj1"] = np.array(m.objective(0, 1))
    for k in ("Omega", "delta", "X", "T", "rho"):
        out["step1_" + k] = m.get(k)
    out.update(extra)
    m.close()
    # an independent fit from the start with a budget of 12 L-BFGS steps
    m = refcpu.RefModel.from_dataset(ds)
    m.set_params(ds.init)
    m.kernel_mats()
    m.glm_init()
    rc, st, tr = m.fit(1, 12)
    out["fit_rc"] = np.array(rc)
    out["fit_stats"] = np.array([st["outer"], st["irls"], st["lbfgs"], st["evals"]])
    out["fit_trace"] = tr
    for k in ("Omega", "delta", "X", "T", "rho", "phi", "Beta"):
        out["fit_" + k] = m.get(k)
    return out


# The DE driver's model comparison (ggplvm_de.cu:886-1207) at parameters from a short
# reference fit: Mfull = the fit's M, Mredc reduced inducing points, budgets of 3 sweeps per
# model and of the driver's own 1000. "de_icpt" has no design variables (the null model is
# the intercept alone, whose first cell the reference's loader sets to 199.0).
DE_CASES = {
    "de_c1": dict(config=1, seed=5, N=300, G=24, M=8, Q=3, Mredc=4),
    "de_icpt": dict(config=0, seed=6, N=250, G=20, M=6, Q=2, Mredc=3, no_vars=True),
}


def make_de_case(name: str, spec: dict) -> dict:
    from gaspacho2_b200.formats import Design

    kw = dict(spec)
    cfg, seed, Mredc = kw.pop("config"), kw.pop("seed"), kw.pop("Mredc")
    no_vars = kw.pop("no_vars", False)
    ds = synth.make(cfg, seed, **kw)
    if no_vars:
        ds.z = Design(ds.N, np.zeros(0, np.int32), np.zeros(0, np.int32), [])
        p = 2
        ds.init.delta = ds.init.delta[[0, -1]].copy()
        assert ds.init.delta.shape[0] == p
    m = refcpu.RefModel.from_dataset(ds)
    m.set_params(ds.init)
    m.kernel_mats()
    m.glm_init()
    m.fit(1, 6)
    prm = type(ds.init)(*(m.get(k).copy() for k in ("Omega", "delta", "X", "T", "rho", "phi")))
    prm.X = prm.X.reshape(ds.Q, ds.N).T.copy()
    prm.T = prm.T.reshape(ds.Q, ds.M).T.copy()
    m.close()
    out = {
        "in_N": np.array(ds.y.N), "in_J": np.array(ds.y.J), "in_M": np.array(ds.M), "in_Q": np.array(ds.Q),
        "in_y_i": ds.y.i, "in_y_p": ds.y.p, "in_y_x": ds.y.x, "in_z_c": ds.z.c, "in_z_v": ds.z.v,
        "in_z_body": np.frombuffer(ds.z.body_bytes(), np.uint8), "in_ls": ds.ls, "in_X0": ds.X0,
        "in_Mredc": np.array(Mredc),
    }
    for k, a in zip(("Omega", "delta", "X", "T", "rho", "phi"), prm.flat()):
        out["in_init_" + k] = a
    for tag, jt in (("j3", 3), ("conv", 1000)):
        bfs, sweeps, beta, phi = refcpu.de_bfs(ds, prm, Mredc, ds.M, jt)
        out[f"de_{tag}_BFs"] = bfs
        out[f"de_{tag}_sweeps"] = np.array(sweeps)
        out[f"de_{tag}_phi"] = phi
        out[f"de_{tag}_beta_full"] = beta
    return out


# The variance-component driver (ggplvm_delta.cu:784-1097): a fit (6 L-BFGS steps of the
# reference) of the design without its last numeric covariate, which has a real effect in
# the counts, then that covariate's variance delta[p-2] refitted on the full design from
# 0.01 under budgets of (3 outer iterations, 100 L-BFGS steps) and (8, 100).
VC_CASES = {
    "vc_c1": dict(config=1, seed=8, N=300, G=24, M=8, Q=2),
}


def make_vc_case(name: str, spec: dict) -> dict:
    import dataclasses

    from gaspacho2_b200.formats import Design

    kw = dict(spec)
    cfg, seed = kw.pop("config"), kw.pop("seed")
    ds = synth.make(cfg, seed, **kw)
    z = ds.z
    assert z.c[-1] == 1
    zfit = Design(z.N, z.c[:-1].copy(), z.v[:-1].copy(), list(z.columns[:-1]))
    dfit = dataclasses.replace(ds, z=zfit, init=dataclasses.replace(ds.init, delta=ds.init.delta[1:].copy()))
    m = refcpu.RefModel.from_dataset(dfit)
    m.set_params(dfit.init)
    m.kernel_mats()
    m.glm_init()
    m.fit(1, 6)
    prm = type(ds.init)(*(m.get(k).copy() for k in ("Omega", "delta", "X", "T", "rho", "phi")))
    prm.X = prm.X.reshape(ds.Q, ds.N).T.copy()
    prm.T = prm.T.reshape(ds.Q, ds.M).T.copy()
    m.close()
    out = {
        "in_N": np.array(ds.y.N), "in_J": np.array(ds.y.J), "in_M": np.array(ds.M), "in_Q": np.array(ds.Q),
        "in_y_i": ds.y.i, "in_y_p": ds.y.p, "in_y_x": ds.y.x, "in_z_c": ds.z.c, "in_z_v": ds.z.v,
        "in_z_body": np.frombuffer(ds.z.body_bytes(), np.uint8), "in_ls": ds.ls, "in_X0": ds.X0,
        "in_init_dg": np.array(0.01),
    }
    for k, a in zip(("Omega", "delta", "X", "T", "rho", "phi"), prm.flat()):
        out["fit_" + k] = a
    for tag, it in (("i3", 3), ("i8", 8)):
        dg, obj = refcpu.vc_fit(ds, prm, 0.01, it, 100)
        out[f"vc_{tag}_dg"] = dg
        out[f"vc_{tag}_obj"] = obj
    return out


# The benchmark's shape at a size the reference's host build finishes in minutes: M = 128
# inducing points, Q = 10 latent dimensions and the 100-donor design (batch 4 levels, 3
# numerics, donor 100 levels: P = 236 model columns, 132 of them dense), with N and G cut.
# The large buffers are kept as a seeded sample of entries (idx_<key>) with the full buffer's
# largest magnitude (scale_<key>); sens_<key> is the reference's own change when X and T move
# by a fraction of an ulp (two perturbed runs), the rounding floor any reordering reaches.
HEAD_CASES = {
    "c2_head": dict(config=2, seed=21, N=2000, G=16, M=128, Q=10),
}
HEAD_SAMPLED = ("kmats_Knm", "kmats_KinvKmn", "sweep0_Psi3", "grad0_C1")


def make_head_case(name: str, spec: dict) -> dict:
    import dataclasses

    sys.path.insert(0, os.path.join(ROOT, "tests"))
    import golden_util as gu  # noqa: E402

    kw = dict(spec)
    cfg, seed = kw.pop("config"), kw.pop("seed")
    ds = synth.make(cfg, seed, **kw)

    def run(d):
        m = refcpu.RefModel.from_dataset(d)
        o = gu.run_phases(m, d)
        m.close()
        m = refcpu.RefModel.from_dataset(d)
        o.update(gu.run_fit(m, d))
        m.close()
        return o

    base = run(ds)
    sens = {}
    same_decisions = True  # the perturbed runs took the same discrete decisions
    for sd in (0, 1):
        rng = np.random.default_rng(sd)
        X2 = ds.init.X * (1 + 2e-16 * rng.standard_normal(ds.init.X.shape))
        T2 = ds.init.T * (1 + 2e-16 * rng.standard_normal(ds.init.T.shape))
        d2 = dataclasses.replace(ds, init=dataclasses.replace(ds.init, X=X2, T=T2))
        pert = run(d2)
        same_decisions &= int(pert["irls_n"]) == int(base["irls_n"]) and \
            np.array_equal(np.asarray(pert["fit_stats"]), np.asarray(base["fit_stats"]))
        for k in base:
            if k not in ("irls_n", "fit_rc", "fit_stats"):
                sens[k] = max(sens.get(k, 0.0), gu.rel_err(np.atleast_1d(pert[k]), np.atleast_1d(base[k])))
    out = {
        "in_N": np.array(ds.y.N), "in_J": np.array(ds.y.J), "in_M": np.array(ds.M), "in_Q": np.array(ds.Q),
        "in_y_i": ds.y.i, "in_y_p": ds.y.p, "in_y_x": ds.y.x, "in_z_c": ds.z.c, "in_z_v": ds.z.v,
        "in_z_body": np.frombuffer(ds.z.body_bytes(), np.uint8), "in_ls": ds.ls, "in_X0": ds.X0,
        "same_decisions": np.array(same_decisions),
    }
    for k, a in zip(("Omega", "delta", "X", "T", "rho", "phi"), ds.init.flat()):
        out["in_init_" + k] = a
    for k, v in base.items():
        v = np.atleast_1d(np.asarray(v))
        if k in HEAD_SAMPLED:
            idx = np.sort(np.random.default_rng(7).choice(v.shape[0], 8192, replace=False))
            out["idx_" + k] = idx.astype(np.int64)
            out["scale_" + k] = np.array(np.abs(v[np.isfinite(v)]).max())
            v = v[idx]
        out[k] = v
        if k in sens:
            out["sens_" + k] = np.array(sens[k])
    return out


def main():
    if not refcpu.available():
        raise SystemExit("build the reference first: make -C oracle ref")
    only = set(sys.argv[1:])
    for name, spec in CASES.items():
        if only and name not in only:
            continue
        out = make_case(name, spec)
        path = os.path.join(OUT, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB, irls sweeps {int(out['irls_n'])}, "
              f"fit {out['fit_stats'].tolist()}")
    for name, spec in HEAD_CASES.items():
        if only and name not in only:
            continue
        out = make_head_case(name, spec)
        path = os.path.join(OUT, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB, irls sweeps {int(out['irls_n'])}, "
              f"fit {out['fit_stats'].tolist()}")
    for name, spec in VC_CASES.items():
        if only and name not in only:
            continue
        out = make_vc_case(name, spec)
        path = os.path.join(OUT, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB, delta_G {out['vc_i8_dg'].tolist()}")
    for name, spec in DE_CASES.items():
        if only and name not in only:
            continue
        out = make_de_case(name, spec)
        path = os.path.join(OUT, f"{name}.npz")
        np.savez_compressed(path, **out)
        print(f"{path}: {os.path.getsize(path) / 1024:.0f} KiB, DE sweeps {out['de_conv_sweeps'].tolist()}")


if __name__ == "__main__":
    main()

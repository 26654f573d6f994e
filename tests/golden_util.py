"""Loads a golden fixture (tests/golden/*.npz) back into the dataset form the models take."""
import dataclasses
import os

import numpy as np

from gaspacho2_b200.formats import Counts, Design, Params

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
CASES = ("c0_small", "c2_cats", "edges")
DE_CASES = ("de_c1", "de_icpt")  # the DE driver's model comparison (make_golden.make_de_case)
VC_CASES = ("vc_c1",)  # the variance-component driver (make_golden.make_vc_case)


def load_vc(name: str):
    """A variance-component fixture: (dataset with the full design, the fit's parameters)."""
    g = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    N, J, M, Q = (int(g[k]) for k in ("in_N", "in_J", "in_M", "in_Q"))
    y = Counts(N, J, g["in_y_i"].astype(np.int32), g["in_y_p"].astype(np.int32), g["in_y_x"])
    c, v = g["in_z_c"].astype(np.int32), g["in_z_v"].astype(np.int32)
    body = g["in_z_body"].tobytes()
    cols, off = [], 0
    for k in range(c.shape[0]):
        nb = (8 if c[k] == 1 else 4) * N * int(v[k])
        if c[k] == 1:
            cols.append(np.frombuffer(body[off:off + nb], np.float64).reshape(int(v[k]), N).T.copy())
        else:
            cols.append(np.frombuffer(body[off:off + nb], np.int32)[:N].copy())
        off += nb
    z = Design(N, c, v, cols)
    prm = Params(g["fit_Omega"], g["fit_delta"], g["fit_X"].reshape(Q, N).T.copy(), g["fit_T"].reshape(Q, M).T.copy(),
                 g["fit_rho"], g["fit_phi"])
    init = Params(g["fit_Omega"], np.zeros(c.shape[0] + 2), prm.X, prm.T, g["fit_rho"], g["fit_phi"])
    ds = GoldenData(y, z, g["in_ls"], g["in_X0"].reshape(N, Q) if g["in_X0"].ndim == 1 else g["in_X0"], init, M, Q, g)
    return ds, prm


@dataclasses.dataclass
class GoldenData:
    y: Counts
    z: Design
    ls: np.ndarray
    X0: np.ndarray
    init: Params
    M: int
    Q: int
    g: dict

    @property
    def N(self):
        return self.y.N

    @property
    def J(self):
        return self.y.J


def load(name: str) -> GoldenData:
    g = dict(np.load(os.path.join(GOLDEN, f"{name}.npz")))
    N, J, M, Q = (int(g[k]) for k in ("in_N", "in_J", "in_M", "in_Q"))
    y = Counts(N, J, g["in_y_i"].astype(np.int32), g["in_y_p"].astype(np.int32), g["in_y_x"])
    c, v = g["in_z_c"].astype(np.int32), g["in_z_v"].astype(np.int32)
    body = g["in_z_body"].tobytes()
    cols, off = [], 0
    for k in range(c.shape[0]):
        if c[k] == 1:
            nb = 8 * N * int(v[k])
            cols.append(np.frombuffer(body[off:off + nb], np.float64).reshape(int(v[k]), N).T.copy())
        else:
            nb = 4 * N * int(v[k])
            cols.append(np.frombuffer(body[off:off + nb], np.int32)[:N].copy())
        off += nb
    z = Design(N, c, v, cols)
    X0 = g["in_X0"].reshape(N, Q) if g["in_X0"].ndim == 2 else g["in_X0"]
    p = c.shape[0] + 2
    init = Params(g["in_init_Omega"], g["in_init_delta"], g["in_init_X"].reshape(Q, N).T,
                  g["in_init_T"].reshape(Q, M).T, g["in_init_rho"], g["in_init_phi"])
    assert init.delta.shape[0] == p
    return GoldenData(y, z, g["in_ls"], np.asarray(X0).reshape(N, Q), init, M, Q, g)


def rel_err(a, b) -> float:
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    if a.shape != b.shape:
        raise AssertionError(f"shape {a.shape} != {b.shape}")
    fin = np.isfinite(b)
    if not np.array_equal(fin, np.isfinite(a)):
        return float("inf")
    if not fin.any():
        return 0.0
    scale = np.abs(b[fin]).max()
    return float(np.abs(a[fin] - b[fin]).max() / (scale if scale > 0 else 1.0))


def run_phases(model, gd: GoldenData) -> dict:
    """The fixture's phase sequence (make_golden.make_case) on any model with the common API."""
    out = {}
    model.set_params(gd.init)
    model.kernel_mats()
    for k in ("Knm", "Kmm", "Kinv", "KinvKmn", "titsias"):
        out["kmats_" + k] = model.get(k)
    model.glm_init()
    out["init_Beta"] = model.get("Beta")
    out["sweep0_lkhd"] = model.irls_sweep(0, 0)
    P = model.P
    out["sweep0_Psi3"] = model.get("Psi")[:3 * P * P]
    for k in ("Beta", "phi", "lkhds"):
        out["sweep0_" + k] = model.get(k)
    out["sweep0_W"] = model.get("W")[: model.N * model.J]
    out["sweep0_Nu"] = model.get("Nu")
    n = model.irls(0, 200)
    out["irls_n"] = n
    out["irls_lkhd"] = model.get("lkhd")[:n]
    for k in ("Beta", "phi"):
        out["irls_" + k] = model.get(k)
    g = getattr(gd, "g", None)
    if g is not None and "score_G" in g:
        out["score_S"] = model.score_stats(g["score_G"])
    out["obj0"] = model.objective_after_irls(0)
    out["obj0_lkhds"] = model.get("lkhds")
    out["grad0"] = model.gradient()
    for k in ("tBeta", "C1", "C2"):
        out["grad0_" + k] = model.get(k)
    model.lbfgs_update(0, 0)
    out["obj1"] = model.objective(0, 1)
    for k in ("Omega", "delta", "X", "T", "rho"):
        out["step1_" + k] = model.get(k)
    return out


def run_fit(model, gd: GoldenData, budget: int = 12) -> dict:
    model.set_params(gd.init)
    model.kernel_mats()
    model.glm_init()
    rc, st, tr = model.fit(1, budget)
    out = {"fit_rc": rc, "fit_stats": np.array([st["outer"], st["irls"], st["lbfgs"], st["evals"]]),
           "fit_trace": tr}
    for k in ("Omega", "delta", "X", "T", "rho", "phi", "Beta"):
        out["fit_" + k] = model.get(k)
    return out


def walk_counts(y: Counts) -> np.ndarray:
    """Dense J x N counts as the reference's merge walk sees them: per gene, the entries are
    consumed in order while each index exceeds the last consumed one and lies in [0, N)."""
    out = np.zeros((y.J, y.N))
    for j in range(y.J):
        last = -1
        for l in range(int(y.p[j]), int(y.p[j + 1])):
            i = int(y.i[l])
            if i <= last or i >= y.N:
                break
            out[j, i] = y.x[l]
            last = i
    return out


def effective_counts(model, gd) -> np.ndarray:
    """Recovers the count each (gene, cell) was matched with from W and nu after one
    W/nu pass: nu = eta + y/W - 1 (matched) or eta - 1 (not), with
    eta = log W - log s - delta_GP * titsias * wt (ggplvm.cu:503-511), rounded to the
    nearest integer (the fixtures hold integer counts)."""
    N, J = gd.y.N, gd.y.J
    W = model.get("W")[: N * J].reshape(J, N)
    nu = model.get("Nu").reshape(J, N)
    delta = model.get("delta")
    tits = model.get("titsias")
    eta = np.log(W) - np.log(gd.ls)[None, :] - delta[-1] * tits[None, :] * 0.1
    return np.rint((nu - eta + 1.0) * W)

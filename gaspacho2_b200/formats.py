"""On-disk formats of the GASPACHO2 driver, read and written byte-compatibly.

Every layout below is the reference's; the citations give the reader/writer it matches.

* counts ``Y.bin`` -- gene-major compressed sparse counts (SparseMat.cu:37-52):
  ``int32 N, J, L; int32 i[L]; int32 p[J+1]; float64 x[L]``.
* design ``Z.bin`` -- the covariate DataFrame (DataFrame.cu:88-149):
  ``int32 N, n_var; int32 c[n_var]; int32 v[n_var]``, then one body block per variable:
  numeric (``c == 1``) ``float64[N*v]`` column-major, categorical (``c > 1``) ``int32[N]``
  level codes in ``0..c-1``. The loader prepends an intercept column and appends the
  M-column Knm block, neither of which is stored in the file.
* size factors ``ls.bin`` -- ``float64[N]`` (ggplvm.cu:1019-1022).
* initial latents ``Xi.bin`` -- ``float64[N*Q]`` column-major (ggplvm.cu:1020-1021).
* parameters ``params.bin`` -- headerless ``float64`` Omega[N], delta[p], X[N*Q], T[M*Q],
  rho[Q], phi[J] (util_cuda.cu:530-535, written by ggplvm.cu:1339-1346).
* checkpoint ``Params9.bin`` -- the same doubles after a 6 x int32 header
  ``N, J, M, P, p, Q`` (util_cuda.cu:566-577).
* ``Tau.bin`` -- ``float64[M*Q]`` (ggplvm.cu:1014).
"""
from __future__ import annotations

import dataclasses
import os
from typing import List, Optional

import numpy as np


@dataclasses.dataclass
class Counts:
    """Gene-major CSR counts: gene j owns entries ``p[j]:p[j+1]`` of ``i`` (cells) and ``x``."""

    N: int
    J: int
    i: np.ndarray  # int32[L]
    p: np.ndarray  # int32[J+1]
    x: np.ndarray  # float64[L]

    @property
    def L(self) -> int:
        return int(self.i.shape[0])


@dataclasses.dataclass
class Design:
    """The file part of a DataFrame: ``n_var`` variables with level counts ``c`` and widths ``v``.

    ``columns[k]`` holds variable k's data: ``float64[N, v]`` for numeric variables,
    ``int32[N]`` level codes for categorical ones.
    """

    N: int
    c: np.ndarray  # int32[n_var]
    v: np.ndarray  # int32[n_var]
    columns: List[np.ndarray]

    @property
    def n_var(self) -> int:
        return int(self.c.shape[0])

    def body_bytes(self) -> bytes:
        parts = []
        for k in range(self.n_var):
            col = self.columns[k]
            if self.c[k] == 1:
                a = np.asarray(col, dtype=np.float64).reshape(self.N, int(self.v[k]))
                parts.append(np.asfortranarray(a).tobytes(order="F"))
            else:
                parts.append(np.asarray(col, dtype=np.int32).reshape(self.N).tobytes())
        return b"".join(parts)

    def model_columns(self, M: int):
        """Column map of the model matrix the reference loader builds (DataFrame.cu:96-134).

        Returns ``(p, P, nh, mc, mv, mk)``: ``p`` variables (intercept + file variables
        + the GP block when M > 0), ``P`` model columns, ``nh[p+1]`` first column of each
        variable, and per column its level count ``mc``, level/sub-column ``mv`` and
        owning variable ``mk``.
        """
        c = [1] + [int(a) for a in self.c] + ([1] if M > 0 else [])
        v = [1] + [int(a) for a in self.v] + ([M] if M > 0 else [])
        p = len(c)
        nh = [0]
        for j in range(p):
            nh.append(nh[-1] + v[j] * c[j])
        P = nh[p]
        mc, mv, mk = [], [], []
        for j in range(p):
            for k in range(nh[j], nh[j + 1]):
                mc.append(c[j])
                mv.append(k - nh[j])
                mk.append(j)
        return p, P, np.array(nh, np.int32), np.array(mc, np.int32), np.array(mv, np.int32), np.array(mk, np.int32)

    def dense_model_matrix(self, M: int, Knm: Optional[np.ndarray] = None) -> np.ndarray:
        """The N x P model matrix Z (getModelMatrix, DataFrame.cu:72-82), Knm block optional."""
        p, P, nh, mc, mv, mk = self.model_columns(M)
        Z = np.zeros((self.N, P))
        Z[:, 0] = 1.0
        for k in range(self.n_var):
            j = k + 1
            col = self.columns[k]
            if self.c[k] == 1:
                Z[:, nh[j]:nh[j + 1]] = np.asarray(col, np.float64).reshape(self.N, -1)
            else:
                codes = np.asarray(col).reshape(self.N)
                for lev in range(int(self.c[k])):
                    Z[:, nh[j] + lev] = (codes == lev).astype(np.float64)
        if M > 0 and Knm is not None:
            Z[:, nh[p - 1]:nh[p]] = Knm
        return Z


@dataclasses.dataclass
class Params:
    """Omega[N], delta[p], X[N, Q] (stored column-major), T[M, Q], rho[Q], phi[J]."""

    Omega: np.ndarray
    delta: np.ndarray
    X: np.ndarray
    T: np.ndarray
    rho: np.ndarray
    phi: np.ndarray

    def flat(self) -> List[np.ndarray]:
        return [
            np.asarray(self.Omega, np.float64).ravel(),
            np.asarray(self.delta, np.float64).ravel(),
            np.asarray(self.X, np.float64).ravel(order="F"),
            np.asarray(self.T, np.float64).ravel(order="F"),
            np.asarray(self.rho, np.float64).ravel(),
            np.asarray(self.phi, np.float64).ravel(),
        ]


def write_counts(path: str, y: Counts) -> None:
    with open(path, "wb") as f:
        np.array([y.N, y.J, y.L], np.int32).tofile(f)
        np.asarray(y.i, np.int32).tofile(f)
        np.asarray(y.p, np.int32).tofile(f)
        np.asarray(y.x, np.float64).tofile(f)


def read_counts(path: str) -> Counts:
    with open(path, "rb") as f:
        N, J, L = (int(a) for a in np.fromfile(f, np.int32, 3))
        i = np.fromfile(f, np.int32, L)
        p = np.fromfile(f, np.int32, J + 1)
        x = np.fromfile(f, np.float64, L)
    if i.shape[0] != L or p.shape[0] != J + 1 or x.shape[0] != L:
        raise ValueError(f"{path}: truncated counts file")
    return Counts(N, J, i, p, x)


def write_design(path: str, z: Design) -> None:
    with open(path, "wb") as f:
        np.array([z.N, z.n_var], np.int32).tofile(f)
        np.asarray(z.c, np.int32).tofile(f)
        np.asarray(z.v, np.int32).tofile(f)
        f.write(z.body_bytes())


def read_design(path: str) -> Design:
    with open(path, "rb") as f:
        N, nv = (int(a) for a in np.fromfile(f, np.int32, 2))
        c = np.fromfile(f, np.int32, nv)
        v = np.fromfile(f, np.int32, nv)
        cols = []
        for k in range(nv):
            if c[k] == 1:
                a = np.fromfile(f, np.float64, N * int(v[k]))
                if a.shape[0] != N * int(v[k]):
                    raise ValueError(f"{path}: truncated design body")
                cols.append(a.reshape(int(v[k]), N).T.copy())
            else:
                a = np.fromfile(f, np.int32, N * int(v[k]))
                if a.shape[0] != N * int(v[k]):
                    raise ValueError(f"{path}: truncated design body")
                cols.append(a[:N].copy())
    return Design(N, c, v, cols)


def write_doubles(path: str, a: np.ndarray, order: str = "C") -> None:
    np.asarray(a, np.float64).ravel(order=order).tofile(path)


def read_doubles(path: str, n: int) -> np.ndarray:
    a = np.fromfile(path, np.float64, n)
    if a.shape[0] != n:
        raise ValueError(f"{path}: expected {n} doubles, found {a.shape[0]}")
    return a


def write_params(path: str, prm: Params, header: Optional[tuple] = None) -> None:
    """``header=(N, J, M, P, p, Q)`` writes the Params9.bin layout, None the params.bin one."""
    with open(path, "wb") as f:
        if header is not None:
            np.array(header, np.int32).tofile(f)
        for a in prm.flat():
            a.tofile(f)


def read_params(path: str, N: int, J: int, M: int, p: int, Q: int, header: bool = False) -> Params:
    with open(path, "rb") as f:
        if header:
            hdr = np.fromfile(f, np.int32, 6)
            if hdr.shape[0] != 6:
                raise ValueError(f"{path}: truncated header")
            N, J, M, _P, p, Q = (int(a) for a in hdr)
        sizes = [N, p, N * Q, M * Q, Q, J]
        parts = []
        for n in sizes:
            a = np.fromfile(f, np.float64, n)
            if a.shape[0] != n:
                raise ValueError(f"{path}: truncated parameter file")
            parts.append(a)
    return Params(parts[0], parts[1], parts[2].reshape(Q, N).T.copy(), parts[3].reshape(Q, M).T.copy(),
                  parts[4], parts[5])


def write_dataset(dirname: str, y: Counts, z: Design, ls: np.ndarray, X0: np.ndarray,
                  init: Optional[Params] = None) -> dict:
    """Writes Y.bin, Z.bin, ls.bin, Xi.bin (and params.bin) as the reference CLI expects."""
    os.makedirs(dirname, exist_ok=True)
    paths = {k: os.path.join(dirname, f"{k}.bin") for k in ("Y", "Z", "ls", "Xi")}
    write_counts(paths["Y"], y)
    write_design(paths["Z"], z)
    write_doubles(paths["ls"], ls)
    write_doubles(paths["Xi"], X0, order="F")
    if init is not None:
        paths["params"] = os.path.join(dirname, "params_init.bin")
        write_params(paths["params"], init)
    return paths

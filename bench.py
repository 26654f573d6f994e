"""Throughput benchmark: objective+gradient evaluations per second of the sparse GP-LVM fit.

One step = one evaluation of the objective and its full gradient at fixed IRLS weights
(kernel matrices, prior, per-gene Gram, batched Cholesky, likelihood, tilde-beta and every
gradient block: d/dlog Omega, d/dlog delta, d/dX, d/dT, d/dlog rho), the unit that the
reference's L-BFGS loop repeats (ggplvm.cu:1215-1277).

Workload (default): 100,000 cells x 10,000 genes, M=128 inducing points, Q=10 latent
dimensions, covariates of the 100-donor configuration (P=236 model columns), seeded
synthetic counts. W and nu (8 GB each) exceed the 126 MB L2, so no flush is needed
between steps.

    python bench.py [--gpus N --steps K --warmup W] [--impl reference]

Under torchrun (N > 1) every rank runs an independent replica on its own GPU (the fit does
not shard across GPUs: one evaluation per rank, no collective on the data path); rank 0
prints one JSON line with the whole-job rate and the slowest rank's device time.
"""
from __future__ import annotations

import argparse
import json
import os
import statistics
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "obj+grad evals/s (100K cells x 10K genes, M=128, Q=10)"
FALLBACK_BF16_SUSTAINED = 1400.0  # TFLOP/s, earlier measurement on this hardware pool
FALLBACK_HBM_GBS = 6650.0  # GB/s, earlier copy measurement on this hardware pool
PEAKS_FILE = os.path.join(ROOT, "MEASURED_PEAKS.json")
# the library's profile ranges (gpl_profile_read names) reported per evaluation
PHASES = ("gram", "uq", "spair", "v_to_u", "whiten", "unwhiten", "split_weights", "split_sdd", "grad_reduce", "chol",
          "inverse", "zt_u", "zbeta", "c1_tn", "kernel_mats", "kinvkmn", "lkhd_genes", "solve", "grad_delta", "c2",
          "grad_tau_rho", "tn_sum", "grad_omega_cell", "oinvt", "collect", "expand_delta", "chol_small", "group_sums",
          "assemble_psi", "assemble_b", "group_tables", "hk", "group_t", "refine", "unwhiten_u", "irls_tail",
          "beta_phi", "lkhd_pois", "w_nu", "logdet_probe")


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--plain", action="store_true",
                    help="time the plain launches (no graphs, separate IRLS tail kernels, no autotuning)")
    ap.add_argument("--profile-steps", type=int, default=1,
                    help="eager evaluations after the timed region for the per-kernel profile")
    ap.add_argument("--no-encoder-leg", action="store_true", help="skip the amortised encoder's experiment")
    ap.add_argument("--enc-config", type=int, default=1)
    ap.add_argument("--enc-train", type=int, default=16384)
    ap.add_argument("--enc-test", type=int, default=4096)
    ap.add_argument("--enc-fit-lbfgs", type=int, default=60)
    ap.add_argument("--enc-epochs", type=int, default=40)
    ap.add_argument("--enc-genes", type=int, default=1000)
    ap.add_argument("--enc-lr", type=float, default=1e-3)
    ap.add_argument("--encoder-report", action="store_true",
                    help="instead of the benchmark: the encoder's experiment alone, once per value of --enc-epochs-list")
    ap.add_argument("--enc-epochs-list", default="",
                    help="comma-separated epoch counts for --encoder-report (default: --enc-epochs)")
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", type=int, default=2)
    ap.add_argument("--N", type=int, default=None)
    ap.add_argument("--G", type=int, default=None)
    ap.add_argument("--precision", default="fp64", choices=["fp64", "bf16x3"])
    ap.add_argument("--irls-sweeps", type=int, default=2)
    ap.add_argument("--option", action="append", default=[],
                    help="name=value: a library option (gpl_set_option) for the benchmark's, the precision leg's "
                         "and the fit-trace contexts; repeatable")
    ap.add_argument("--eta-tc", type=int, default=None,
                    help="option eta_tc (linear predictor and W / Nu on the FP64 tensor cores): 0 or 1; "
                         "default: the library's")
    ap.add_argument("--cpu-genes", type=int, default=6, help="genes in the bounded CPU sample")
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--fit-config", type=int, default=1, help="configuration of the time-to-fit leg")
    ap.add_argument("--fit-lbfgs", type=int, default=200, help="L-BFGS step budget of the time-to-fit leg")
    ap.add_argument("--no-fit", action="store_true", help="skip the time-to-fit leg")
    ap.add_argument("--no-precision-leg", action="store_true",
                    help="skip the precision form's throughput beside the FP64 line")
    ap.add_argument("--precision-report", action="store_true",
                    help="instead of the benchmark: the precision form against FP64 along a fit, every 10 steps")
    ap.add_argument("--no-de-leg", action="store_true",
                    help="skip the DE driver's model-comparison pass beside the FP64 line")
    ap.add_argument("--de-mredc", type=int, default=5, help="inducing points of the DE per-dimension models")
    ap.add_argument("--reference-gpu", action="store_true",
                    help="instead of the benchmark: the reference's own CUDA build against this project's "
                         "evaluation on --config (use --config 0)")
    ap.add_argument("--ref-gpu-steps", type=int, default=20)
    ap.add_argument("--ref-gpu-seconds", type=float, default=240.0)
    ap.add_argument("--fit-trace", action="store_true",
                    help="instead of the benchmark: the --fit-config fit per outer iteration, each precision of "
                         "--fit-precisions")
    ap.add_argument("--fit-precisions", default="fp64,bf16x3")
    ap.add_argument("--fit-max-outer", type=int, default=1000)
    ap.add_argument("--slope-check", action="store_true",
                    help="instead of the benchmark: at the state after the second outer iteration's IRLS of "
                         "--fit-config, each form's objective slope along the unit gradient direction against "
                         "its gradient, and the precision form's errors per block, with and without the "
                         "log-determinant probe")
    ap.add_argument("--fit-spread", action="store_true",
                    help="instead of the benchmark: the --fit-config fit's end point from starts perturbed by "
                         "1e-12 and 1e-9 (relative, X), FP64 and the precision form")
    return ap.parse_args()


# ---- clocks ------------------------------------------------------------------------------------
class ClockSampler:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device: int):
        self.device = device
        self.proc = None
        self.path = None

    def start(self):
        fd, self.path = tempfile.mkstemp(prefix="clocks_", suffix=".csv")
        os.close(fd)
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.device}", f"--query-gpu={self.FIELDS}", "--format=csv,noheader,nounits",
                 "-lms", "200"], stdout=open(self.path, "w"), stderr=subprocess.DEVNULL)
        except OSError:
            self.proc = None

    def stop(self) -> dict:
        if self.proc is None:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(timeout=5)
        except subprocess.TimeoutExpired:
            self.proc.kill()
        sm, smax, reasons = [], [], set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            parts = [x.strip() for x in line.split(",")]
            if len(parts) < 9:
                continue
            try:
                sm.append(float(parts[1]))
                smax.append(float(parts[2]))
            except ValueError:
                continue
            for nm, v in zip(names, parts[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        os.unlink(self.path)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": max(smax) if smax else None,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_peaks():
    try:
        with open(PEAKS_FILE) as f:
            return json.load(f)
    except OSError:
        return {}


_FP64_PEAK = []


def fp64_peak_tflops(torch) -> float:
    """Dense FP64 GEMM rate on this GPU (torch.matmul float64 8192^3, best of 5), the FP64
    counterpart of the bf16 figure in MEASURED_PEAKS.json, which has no FP64 entry; measured
    once per run."""
    if _FP64_PEAK:
        return _FP64_PEAK[0]
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device="cuda")
    b = torch.randn(n, n, dtype=torch.float64, device="cuda")
    torch.matmul(a, b)
    torch.cuda.synchronize()
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        e.synchronize()
        best = min(best, s.elapsed_time(e) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    _FP64_PEAK.append(2.0 * n ** 3 / best / 1e12)
    return _FP64_PEAK[0]


def flops_table(N, J, M, P, n_dense):
    """Algorithmic flops per launch of the dominant kernels (2 flops per multiply-add)."""
    return {
        # Gram over the dense model columns: n_d*(n_d+1)/2 unique pairs, 2 flops per cell and gene
        "gram": float(N) * J * n_dense * (n_dense + 1),
        # gradient contraction sum_j O_ij S_j[DD] d_i over the unique pairs of the symmetric S_j
        # (the pair form's V = O S_pairs; the epilogue to U is N*n_d^2, not counted)
        "uq": float(N) * J * n_dense * (n_dense + 1),
        # the cell x gene FP64 GEMMs around them (per launch)
        "zt_u": 2.0 * N * J * n_dense,
        "group_sums": 2.0 * N * J * n_dense,
        "hk": 2.0 * N * J * (n_dense + 1),
        "c1_tn": 2.0 * N * J * M,
        # batched SPD inverse (triangular inverse + its product, n^3/3 flops each) and Cholesky
        "inverse": 2.0 / 3.0 * J * float(P) ** 3,
        "chol": 1.0 / 3.0 * J * float(P) ** 3,
    }


# ---- CPU legs: bounded samples of the same workload --------------------------------------------
class CpuSample:
    """A bounded sample of the workload on the host cores: the first `genes` genes with all
    cells, through the reference's own kernels built for the host (oracle/_ref, "reference")
    or, where that build is absent, the oracle's restatement ("port"). One step is one
    objective + gradient evaluation. Its time is split into a gene-independent part (the kernel
    matrices and the cell x inducing-point terms of the gradient) and a part linear in the
    genes, measured once at setup from steps at `genes` (the faster of two) and at 2 * `genes`
    genes (t(2g) - t(g) is the per-gene part of g genes); each step's time is then the fixed
    part plus its per-gene part scaled to all genes."""

    def __init__(self, ds, genes: int):
        from gaspacho2_b200 import synth
        from oracle import port, refcpu

        self.threads = os.cpu_count() or 1
        self.kind = "reference" if refcpu.available() else "port"
        if self.kind == "port":
            port.set_threads(self.threads)

        def model(g):
            sub = synth.gene_subset(ds, g)
            m = refcpu.RefModel.from_dataset(sub) if self.kind == "reference" else port.OracleModel.from_dataset(sub)
            m.set_params(sub.init)
            m.kernel_mats()
            m.glm_init()
            m.irls_sweep(0, 0)
            m.objective_after_irls(0)
            return sub, m

        self.sub, self.m = model(genes)
        self.slot = 1
        t1 = min(self._raw(), self._raw())
        _, m2 = model(2 * genes)
        t0 = time.perf_counter()
        m2.gradient()
        m2.objective(0, 1)
        t2 = time.perf_counter() - t0
        del m2
        self.fixed = min(max(2.0 * t1 - t2, 0.0), t1)
        self.scale = ds.J / float(genes)
        self.desc = (f"{genes} of {ds.J} genes with all {ds.N} cells, one objective+gradient evaluation per step "
                     f"on {self.threads} host threads; the step's gene-independent part ({self.fixed:.2f} s, from "
                     f"one step at {genes} and one at {2 * genes} genes: {t1:.2f} s, {t2:.2f} s) plus its "
                     f"per-gene part scaled by {self.scale:.0f} to all genes")

    def _raw(self) -> float:
        t0 = time.perf_counter()
        self.m.gradient()
        self.m.objective(0, self.slot)
        self.slot += 1
        return time.perf_counter() - t0

    def step(self) -> float:
        t = self._raw()
        return self.fixed + max(t - self.fixed, 0.0) * self.scale


PARITY_TOL = 1e-8  # per-buffer relative error of the FP64 path against the reference's kernels


def bench_parity(cs, device, stream):
    """The CUDA path against the reference's kernels built for the host at the bench's shape:
    the CPU sample's genes with all cells (M, Q, P and the cell ranges of the full workload),
    the same call sequence on a context over those genes (GLM initialisation, one IRLS sweep,
    the objective, then one gradient and one objective as the CPU step runs them), compared
    per gene (the Laplace objective pieces l_j, tilde-beta_j, the diagonal of each factored
    Psi_j) and on the whole gradient (every cell-summed block over those genes) and the
    objective. Errors are max |a - b| / max |b| per buffer."""
    from gaspacho2_b200 import GPLVM

    sub, ref = cs.sub, cs.m
    with GPLVM.from_dataset(sub, device=device, stream=stream.cuda_stream, precision="fp64") as m:
        m.set_params(sub.init)
        m.kernel_mats()
        m.glm_init()
        m.irls_sweep(0, 0)
        m.objective_after_irls(0)
        g = m.gradient()
        v = m.objective(0, 1)
        P, J = m.P, m.J
        got = {"objective": np.array([v]), "grad": g, "lkhds": m.get("lkhds"), "tBeta": m.get("tBeta"),
               "Psi_diag": m.get("Psi").reshape(J, P, P)[:, np.arange(P), np.arange(P)].ravel()}
    want = {"objective": np.array([ref.get("lkhd")[cs.slot - 1]]), "grad": ref.get("grad")[:g.shape[0]],
            "lkhds": ref.get("lkhds"), "tBeta": ref.get("tBeta"),
            "Psi_diag": ref.get("Psi")[:J * P * P].reshape(J, P, P)[:, np.arange(P), np.arange(P)].ravel()}
    errs = {}
    for k in got:
        a, b = np.asarray(got[k], np.float64), np.asarray(want[k], np.float64)
        fin = np.isfinite(b)
        errs[k] = float("inf") if not np.array_equal(fin, np.isfinite(a)) else \
            float(np.abs(a[fin] - b[fin]).max() / max(np.abs(b[fin]).max(), 1e-300))
    return {"against": f"the reference's kernels built for the host ({cs.kind}), same state and call sequence",
            "genes": int(J), "cells": int(sub.N), "max_rel_err": errs, "tol": PARITY_TOL,
            "pass": bool(all(e <= PARITY_TOL for e in errs.values()))}


def dataset(args):
    from gaspacho2_b200 import synth

    kw = {}
    if args.N:
        kw["N"] = args.N
    if args.G:
        kw["G"] = args.G
    return synth.make(args.config, 0, init=False, **kw)


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    ds = dataset(args)
    cs = CpuSample(ds, args.cpu_genes)
    per_eval = []
    for i in range(args.warmup + args.steps):
        t = cs.step()
        if i >= args.warmup:
            per_eval.append(t)
    kind, threads, desc = cs.kind, cs.threads, cs.desc
    t = statistics.mean(per_eval)
    value = 1.0 / t
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": t * 1e3, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(ds, args, "fp64"),
        "cpu_baseline": {"value": value, "unit": "evals/s", "cores": threads, "kind": kind, "sample": desc},
        "e2e": {"value": value, "unit": "evals/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def workload_config(ds, args, precision):
    p = ds.z.n_var + 2
    M, Q = ds.M, ds.Q
    P = 1 + int(sum(int(c) * int(v) for c, v in zip(ds.z.c, ds.z.v))) + M
    return {"workload": f"config {args.config}: N={ds.N} cells, G={ds.J} genes, M={M}, Q={Q}, P={P}, p={p}",
            "N": ds.N, "G": ds.J, "M": M, "Q": Q, "P": P, "precision": precision,
            "l2": "inputs larger than L2 (W and nu are N*G doubles each)", "parallelism": f"replicas{args.gpus}",
            "global_batch": ds.N, "seq_len": None}


def de_leg(args, ds, stream, device):
    """The DE driver's model comparison (ggplvm_de.cu:1067-1207) on the bench workload: one pass
    of its table, i.e. the GLM initialisation and one IRLS sweep of each of the Q + 2 models
    (null, the GP over each latent dimension with --de-mredc equispaced points, the full GP),
    at the workload's starting parameters. Timed with CUDA events on the library's stream
    around `de.de_bfs(jtr_max=1)` on contexts opened beforehand (one warm-up pass). The CPU
    baseline runs the same pass through the oracle on 8 and 16 genes with all cells and
    extrapolates linearly in the gene count (the kernel matrices and the single initial
    factorisation do not grow with genes)."""
    import torch

    from gaspacho2_b200 import de

    Mr = args.de_mredc
    ctxs = de.open_contexts(ds.y, ds.z, ds.ls, ds.init.X, ds.Q, Mr, ds.M, device, stream.cuda_stream)
    try:
        de.de_bfs(ds.y, ds.z, ds.ls, ds.init, ds.Q, Mr, ds.M, 1, contexts=ctxs)
        torch.cuda.synchronize()
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record(stream)
        out = de.de_bfs(ds.y, ds.z, ds.ls, ds.init, ds.Q, Mr, ds.M, 1, contexts=ctxs)
        e.record(stream)
        torch.cuda.synchronize()
        t = s.elapsed_time(e) / 1e3
    finally:
        for m in ctxs:
            m.close()
    res = {"metric": "DE model-table passes/s (GLM init + 1 IRLS sweep of each of the Q+2 models)",
           "value": 1.0 / t, "unit": "passes/s", "seconds_per_pass": t, "models": ds.Q + 2, "Mredc": Mr,
           "Mfull": ds.M, "dtype": "f64", "finite": bool(np.all(np.isfinite(out["BFs"])))}
    if not args.no_cpu_baseline:
        from gaspacho2_b200 import synth
        from oracle import port

        # the oracle's restatement (bit-exact with the reference's DE kernels on the golden
        # cases): the reference's own null model reads level codes out of range when the last
        # design variable is categorical, as it is here (the donor), so it cannot run this design
        threads = os.cpu_count() or 1
        port.set_threads(threads)
        ts = {}
        for g in (8, 16):
            sub = synth.gene_subset(ds, g)
            t0 = time.perf_counter()
            port.de_bfs(sub, sub.init, Mr, ds.M, 1)
            ts[g] = time.perf_counter() - t0
        slope = (ts[16] - ts[8]) / 8.0
        t_cpu = max(ts[16] + slope * (ds.J - 16), ts[16])
        res["cpu_baseline"] = {"value": 1.0 / t_cpu, "unit": "passes/s", "cores": threads, "kind": "port",
                               "sample": f"8 and 16 of {ds.J} genes with all {ds.N} cells ({ts[8]:.1f} s, "
                                         f"{ts[16]:.1f} s), linear in genes to all {ds.J}"}
    return res


# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) of one Gram (the pair products
# written once, then the GEMM), from a single-pass ncu capture of this bench's own command at
# config 2 (the metric is not available inside the timed run): k_pair_products read 0.11 GB and
# wrote 7.00 GB, k_pair_gram read 174.40 GB and wrote 1.73 GB, against 16.6 GB of algorithmic
# bytes (products 7.1 GB written and read once, W 8.0 GB read, Psi dense blocks 1.4 GB written):
# the grouped tile order leaves each operand tile read from DRAM about 11 times, at 0.3 TB/s.
TRAFFIC_BYTES = {("gram", 2, 100000, 10000, 128, 10): 0.11e9 + 7.00e9 + 174.40e9 + 1.73e9}


def measured_traffic(kernel, ds, args):
    return TRAFFIC_BYTES.get((kernel, args.config, ds.N, ds.J, ds.M, ds.Q))


def irls_leg(m, ds, args, stream, torch):
    """IRLS sweeps (getWForBeta, getPsi, cholPsi, getBetaPhi, getLkhdPois: ggplvm.cu:1156-1181)
    at the bench state: 3 sweeps timed with CUDA events, their phases from the library's
    profile, and the W / nu kernel against its two bounds: the HBM bytes it must move (W and
    nu written, the counts and dense columns read) at the measured copy bandwidth, and the
    FP64 multiply-adds of the linear predictor (2 N J n_d) at the measured FP64 GEMM rate; the
    larger of the two times is the bound it is measured against."""
    m.profile(True)
    m.profile_reset()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    n = 3
    s.record(stream)
    for j in range(n):
        m.irls_sweep(0, args.irls_sweeps + j)
    e.record(stream)
    torch.cuda.synchronize()
    t = s.elapsed_time(e) / 1e3 / n
    ph = {}
    for name in ("w_nu", "gram", "group_sums", "assemble_psi", "chol", "zt_u", "solve", "beta_phi", "lkhd_pois",
                 "collect"):
        ms, k = m.profile_read(name)
        if k:
            ph[name] = ms / n
    m.profile(False)
    N, J, n_d = m.N, m.J, m.n_dense()
    nnz = int(ds.y.L)
    bytes_w_nu = 2.0 * 8 * N * J + 12.0 * nnz + 8.0 * N * n_d + 8.0 * N
    flops_w_nu = 2.0 * N * J * n_d
    hbm = (measured_peaks().get("hbm_gbs") or FALLBACK_HBM_GBS) * 1e9
    f64 = fp64_peak_tflops(torch) * 1e12
    t_w = ph.get("w_nu", 0.0) / 1e3
    bound = "hbm" if bytes_w_nu / hbm >= flops_w_nu / f64 else "fp64"
    t_bound = max(bytes_w_nu / hbm, flops_w_nu / f64)
    return {"ms_per_sweep": t * 1e3, "phase_ms_per_sweep": ph,
            "w_nu_roofline": {"bound": bound, "algorithmic_bytes": bytes_w_nu, "flops": flops_w_nu,
                              "achieved_gbs": bytes_w_nu / t_w / 1e9 if t_w else None,
                              "achieved_tflops": flops_w_nu / t_w / 1e12 if t_w else None,
                              "frac": t_bound / t_w if t_w else None,
                              "note": "bound = the larger of bytes / measured copy bandwidth and flops / measured "
                                      "FP64 GEMM rate; frac = that time / the kernel's time"}}


def grad_blocks(g, ref, N, p, Q, M):
    """Relative L2 error of g against ref per block of the parameter vector
    [log Omega (N) | log delta (p) | X (N Q) | T (M Q) | log rho (rest)]."""
    edges = np.cumsum([0, N, p, N * Q, M * Q, len(ref) - (N + p + N * Q + M * Q)])
    out = {}
    for name, a, b in zip(("log_omega", "log_delta", "X", "T", "log_rho"), edges[:-1], edges[1:]):
        if b > a:
            out[name] = float(np.linalg.norm(g[a:b] - ref[a:b]) / max(np.linalg.norm(ref[a:b]), 1e-300))
    return out


def precision_leg(args, ds, stream, device):
    """The precision form (tensor-core Gram and gradient contraction over whitened columns,
    FP64 elsewhere, refined solves) on the same workload and state as the FP64 line: its
    device-resident evaluation rate, and its objective and gradient against FP64 at the
    same parameters."""
    import torch

    from gaspacho2_b200 import GPLVM

    m = GPLVM.from_dataset(ds, device=device, stream=stream.cuda_stream, precision="fp64")
    m.set_params(ds.init)
    m.kernel_mats()
    m.glm_init()
    for j in range(args.irls_sweeps):
        m.irls_sweep(0, j)
    m.objective_after_irls(0)
    x = m.params_vector()
    v64, g64 = m.evaluate(x)
    g64 = g64.copy()
    m.set_precision("bf16x3")
    vbf, gbf = m.evaluate(x)
    gbf = gbf.copy()
    batched = not args.plain
    if args.eta_tc is not None:
        m.set_option("eta_tc", args.eta_tc)
    for kv in args.option:
        k, v = kv.split("=")
        m.set_option(k, int(v))
    if batched:
        for k in ("autotune", "graph"):
            m.set_option(k, 1)
    warm = 0
    while warm < args.warmup or (batched and warm < 30 and m.get_option("graph_replays") < 2 and
                                 m.get_option("graph") == 1):
        m.evaluate_device()
        m.sync()
        warm += 1
    torch.cuda.synchronize()
    r0 = m.get_option("graph_replays")
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(args.steps):
        m.evaluate_device()
    e.record(stream)
    torch.cuda.synchronize()
    dt = s.elapsed_time(e) / 1e3
    replays = m.get_option("graph_replays") - r0
    m.profile(True)
    m.profile_reset()
    for _ in range(args.profile_steps):
        m.evaluate_device()
    torch.cuda.synchronize()
    phases = {}
    for name in PHASES:
        ms, n = m.profile_read(name)
        if n:
            phases[name] = ms / args.profile_steps
    m.profile(False)
    tuning = {k: m.tuning(k) for k in ("tc_gram", "tc_grad", "eta_tile")} if batched else None
    m.close()
    return {"value": args.steps / dt, "unit": "evals/s", "ms_per_step": dt / args.steps * 1e3,
            "dtype": "bf16x3+f64", "objective_rel_err_vs_fp64": abs(vbf - v64) / abs(v64),
            "gradient_rel_l2_vs_fp64": float(np.linalg.norm(gbf - g64) / np.linalg.norm(g64)),
            "gradient_rel_l2_by_block": grad_blocks(gbf, g64, ds.N, len(ds.init.delta), ds.Q, ds.M),
            "graph_replays_timed": int(replays), "autotune": tuning,
            "phase_ms_per_step": phases,
            "phase_note": f"per-kernel CUDA-event times of {args.profile_steps} eager evaluations after the timed region",
            "note": "Gram and gradient contraction on tcgen05 (BF16 hi/lo, FP64-folded TMEM runs) over "
                    "whitened dense columns; FP64 elsewhere; one FP64-residual refinement per solve"}


def time_to_fit(args, stream, device):
    """The driver's whole fit (kernel matrices, GLM initialisation, then outer iterations of
    IRLS to convergence and L-BFGS with the backtracking line search) from the seeded
    PCA / k-means initialisation, up to the L-BFGS step budget, timed with CUDA events on the
    library's stream (the line-search decisions read the objective on the host, as in the
    reference driver, so this is also the wall time)."""
    import torch

    from gaspacho2_b200 import GPLVM, synth

    ds = synth.make(args.fit_config, 0, init=True)
    m = GPLVM.from_dataset(ds, device=device, stream=stream.cuda_stream, precision=args.precision)
    m.set_params(ds.init)
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    t0 = time.time()
    s.record(stream)
    m.kernel_mats()
    m.glm_init()
    rc, st, trace = m.fit(100000, args.fit_lbfgs)
    e.record(stream)
    torch.cuda.synchronize()
    wall = time.time() - t0
    secs = s.elapsed_time(e) / 1e3
    m.close()
    cfg = synth.CONFIGS[args.fit_config]
    return {"seconds": secs, "wall_seconds": wall, "lbfgs_budget": args.fit_lbfgs,
            "workload": f"config {args.fit_config}: N={ds.N} cells, G={ds.J} genes, M={ds.M}, Q={ds.Q}, "
                        f"seeded PCA/k-means initialisation",
            "precision": args.precision, "outer_iterations": st["outer"], "irls_sweeps": st["irls"],
            "lbfgs_steps": st["lbfgs"], "objective_evaluations": st["evals"],
            "final_objective": float(trace[-1]) if len(trace) else None, "nan_exit": bool(rc),
            "batch_levels": cfg.get("batch"), "donors": cfg.get("donors")}


def run_ours(args):
    import torch

    from gaspacho2_b200 import GPLVM
    from gaspacho2_b200.replicas import Replicas

    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    rep = Replicas("nccl")  # one independent replica per GPU; barrier and max-over-ranks time only
    world, rank, local = rep.world, rep.rank, rep.local

    ds = dataset(args)
    # a dedicated stream: the library runs every kernel on it and the CUDA events below are
    # recorded on it (torch's default stream has handle 0, which the C ABI reads as "own stream")
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    m = GPLVM.from_dataset(ds, device=local, stream=stream.cuda_stream, precision=args.precision)
    batched = not args.plain
    if args.eta_tc is not None:
        m.set_option("eta_tc", args.eta_tc)
    for kv in args.option:
        k, v = kv.split("=")
        m.set_option(k, int(v))
    if batched:
        # the batched form: the IRLS tail as one persistent launch, evaluations replayed from
        # captured CUDA graphs, tile orders chosen by the autotuner (all give the plain path's bits)
        for k in ("fused_tail", "autotune", "graph"):
            m.set_option(k, 1)
    m.set_params(ds.init)
    m.kernel_mats()
    m.glm_init()
    # with the batched form, enough sweeps for the fused tail's CTA count to be timed and chosen
    for j in range(max(args.irls_sweeps, 4) if batched else args.irls_sweeps):
        m.irls_sweep(0, j)
    m.objective_after_irls(0)
    warm = 0
    while warm < args.warmup or (batched and warm < 40 and m.get_option("graph_replays") < 2 and
                                 m.get_option("graph") == 1):
        m.evaluate_device()
        m.sync()
        warm += 1
    torch.cuda.synchronize()

    barrier = rep.barrier

    # device-resident throughput
    clocks = ClockSampler(local)
    clocks.start()
    l0 = m.launches()
    r0 = m.get_option("graph_replays")
    barrier()
    torch.cuda.synchronize()
    s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s.record(stream)
    for _ in range(args.steps):
        m.evaluate_device()
    e.record(stream)
    torch.cuda.synchronize()
    barrier()
    dt = s.elapsed_time(e) / 1e3
    launches = m.launches() - l0
    replays = m.get_option("graph_replays") - r0
    ck = clocks.stop()
    # per-kernel device times: the same evaluation run eagerly with CUDA events around each kernel
    # (profiling runs outside the graphs), after the timed region
    m.profile(True)
    m.profile_reset()
    s3, e3 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s3.record(stream)
    for _ in range(args.profile_steps):
        m.evaluate_device()
    e3.record(stream)
    torch.cuda.synchronize()
    eager_ms = s3.elapsed_time(e3) / args.profile_steps
    prof = {}
    for name in PHASES:
        ms, n = m.profile_read(name)
        if n:
            prof[name] = (ms, n)
    m.profile(False)
    t_max = rep.max_time(dt)
    value = world * args.steps / t_max

    # end to end through the C ABI with host buffers (pinned), copies inside the timed region
    n_par = m.n_params()
    params = torch.empty(n_par, dtype=torch.float64, pin_memory=True).numpy()
    params[:] = m.params_vector()
    grad = torch.empty(n_par, dtype=torch.float64, pin_memory=True).numpy()
    barrier()
    torch.cuda.synchronize()
    s2, e2 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
    s2.record(stream)
    for _ in range(args.steps):
        m.evaluate(params, grad)
    e2.record(stream)
    torch.cuda.synchronize()
    barrier()
    dt2 = rep.max_time(s2.elapsed_time(e2) / 1e3)
    e2e = {"value": world * args.steps / dt2, "unit": "evals/s", "h2d_bytes_per_step": int(params.nbytes),
           "d2h_bytes_per_step": int(grad.nbytes + 8)}

    irls = irls_leg(m, ds, args, stream, torch) if rank == 0 else None

    line = None
    if rank == 0:
        total_prof = sum(v[0] for v in prof.values())
        dom = max(prof, key=lambda k: prof[k][0])
        P = m.P
        ft = flops_table(m.N, m.J, m.M, P, m.n_dense())
        peaks = measured_peaks()
        tc_kernels = ("gram", "uq") if m.get_option("tc_grad") else ("gram",)
        if dom in ft and args.precision == "bf16x3" and dom in tc_kernels:
            # useful flops of the contraction; the hi/lo split issues 3 BF16 products per useful MAC
            tflops = ft[dom]
            pk = peaks.get("bf16_tflops_sustained") or FALLBACK_BF16_SUSTAINED
            avg_s = prof[dom][0] / prof[dom][1] / 1e3
            achieved = tflops / avg_s / 1e12
            roof = {"kernel": dom, "bound": "tensor", "achieved": achieved, "peak": pk, "unit": "TFLOP/s",
                    "frac": achieved / pk, "traffic": None,
                    "peak_source": ("of measured: bf16_tflops_sustained (cuBLAS bf16 GEMM under the power cap)"
                                    if peaks.get("bf16_tflops_sustained") else "of fallback: 1.4 PFLOP/s sustained"),
                    "flops_per_launch": tflops, "flops_note": "useful flops of the contraction, padding "
                    "excluded; the tensor pipe executes 3x this (hi*hi + hi*lo + lo*hi BF16 products)",
                    "avg_launch_ms": avg_s * 1e3, "share_of_step": prof[dom][0] / max(total_prof, 1e-30)}
        elif dom in ft:
            f64 = fp64_peak_tflops(torch)
            avg_s = prof[dom][0] / prof[dom][1] / 1e3
            achieved = ft[dom] / avg_s / 1e12
            roof = {"kernel": dom, "bound": "tensor", "pipe": "FP64 DMMA (mma.sync.m16n8k4.f64 on the tensor cores)",
                    "achieved": achieved, "peak": f64, "unit": "TFLOP/s",
                    "frac": achieved / f64, "traffic": measured_traffic(dom, ds, args),
                    "peak_source": "measured in this run: torch.matmul float64 8192^3 best of 5 "
                                   "(MEASURED_PEAKS.json has no FP64 entry)",
                    "flops_per_launch": ft[dom], "avg_launch_ms": avg_s * 1e3,
                    "share_of_step": prof[dom][0] / max(total_prof, 1e-30)}
        else:
            roof = {"kernel": dom, "bound": None, "achieved": None, "peak": None, "unit": None, "frac": None,
                    "traffic": None}
        line = {
            "metric": METRIC, "value": value, "unit": "evals/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": t_max / args.steps * 1e3, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if args.precision == "fp64" else "bf16x3+f64",
            "data": "synthetic", "config": workload_config(ds, args, args.precision), "e2e": e2e,
            "gpu_launches": int(launches), "roofline": roof, "clocks": ck,
            "phase_ms_per_step": {k: v[0] / args.profile_steps
                                  for k, v in sorted(prof.items(), key=lambda kv: -kv[1][0])},
            "phase_note": f"per-kernel CUDA-event times of {args.profile_steps} eager evaluations after the timed "
                          f"region ({eager_ms:.1f} ms each, profiling on)",
            "hbm_gbs_measured": peaks.get("hbm_gbs"), "bf16_tflops_measured": peaks.get("bf16_tflops"),
            "irls_sweep": irls,
            "batched_form": {"graph": bool(m.get_option("graph")), "graph_replays_timed": int(replays),
                             "fused_tail": bool(m.get_option("fused_tail")),
                             "autotune": {k: m.tuning(k) for k in ("pair_gram", "pair_v", "irls_tail", "eta_tile")},
                             "eager_profiled_ms_per_step": eager_ms, "warmup_evaluations": warm} if batched else None,
        }
    if rank == 0 and getattr(ds, "genotypes", None) is not None:
        # per-(gene, variant) cis statistics at the bench state (the workload's donor genotypes)
        D, J, V = ds.genotypes.shape
        torch.cuda.synchronize()
        t0 = time.time()
        S, LR = m.cis_stats(ds.genotypes, len(ds.z.c) - 1)
        tc = time.time() - t0
        truth = ds.geno_truth
        causal = LR[np.arange(J), truth["causal"]]
        mask = np.ones_like(LR, bool)
        mask[np.arange(J), truth["causal"]] = False
        line["cis_statistics"] = {"genes": J, "variants_per_gene": V, "donors": D, "seconds": tc,
                                  "median_lr_causal": float(np.median(causal)),
                                  "median_lr_other": float(np.median(LR[mask])),
                                  "finite": bool(np.all(np.isfinite(S))),
                                  "note": "timed at the benchmark's state, whose IRLS has run only the bench's sweeps "
                                          "(not converged), so the values are not calibrated there; the causal "
                                          "variants' separation is tested at convergence (tests/test_gpu_cis.py)"}
    m.close()
    if rank == 0 and world == 1 and not args.no_encoder_leg:
        from gaspacho2_b200.encoder import amortised_placement

        line["encoder"] = amortised_placement(args.enc_config, args.enc_train, args.enc_test, args.enc_fit_lbfgs,
                                              args.enc_epochs, n_genes=args.enc_genes, device=local,
                                              stream=stream.cuda_stream, lr=args.enc_lr)
    if rank == 0 and args.precision == "fp64" and not args.no_precision_leg:
        line["precision_form"] = precision_leg(args, ds, stream, local)
    if rank == 0 and args.precision == "fp64" and not args.no_de_leg:
        line["de_model_comparison"] = de_leg(args, ds, stream, local)
    if rank == 0 and not args.no_fit:
        line["time_to_fit"] = time_to_fit(args, stream, local)
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cs = CpuSample(ds, args.cpu_genes)
        t = cs.step()
        line["cpu_baseline"] = {"value": 1.0 / t, "unit": "evals/s", "cores": cs.threads, "kind": cs.kind,
                                "sample": cs.desc}
        line["parity"] = bench_parity(cs, local, stream)
    if rank == 0:
        print(json.dumps(line), flush=True)
    rep.close()
    return 0


def slope_check(args):
    """The precision form's objective against its gradient: the fit of --fit-config (precision form)
    for one outer iteration of at most 30 L-BFGS steps, the next IRLS, then at that state each form's
    objective and gradient, and finite differences (v(x + eps d) - v(x)) / eps along the unit FP64
    gradient direction d, taken in the gradient's coordinates (log Omega, log delta, X, T, log rho),
    against g . d. One JSON line per setting of the log-determinant probe."""
    import torch

    from gaspacho2_b200 import GPLVM, synth

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    ds = synth.make(args.fit_config, 0, init=True)
    N, Q, M, p = ds.N, ds.Q, ds.M, len(ds.init.delta)
    e = np.cumsum([0, N, p, N * Q, M * Q])
    names = ("log_omega", "log_delta", "X", "T", "log_rho")
    spans = list(zip(e[:-1], e[1:])) + [(e[-1], None)]

    def move(x, d, eps):
        y = x.copy()
        for n, (a, b) in zip(names, spans):
            y[a:b] = x[a:b] * np.exp(eps * d[a:b]) if n.startswith("log_") else x[a:b] + eps * d[a:b]
        return y

    with GPLVM.from_dataset(ds, stream=stream.cuda_stream, precision="bf16x3") as m:
        m.set_params(ds.init)
        m.kernel_mats()
        m.glm_init()
        m.fit_outer(0, 30)
        m.irls(1, 100)
        m.objective_after_irls(1)
        x = m.params_vector()
        m.set_precision("fp64")
        vf, gf = m.evaluate(x)
        gf = gf.copy()
        d = gf / np.linalg.norm(gf)
        for probe in (1, 0):
            m.set_option("logdet_probe", probe)
            m.set_precision("bf16x3")
            vb, gb = m.evaluate(x)
            gb = gb.copy()
            errs = {n: float(np.linalg.norm(gb[a:b] - gf[a:b]) / max(np.linalg.norm(gf[a:b]), 1e-300))
                    for n, (a, b) in zip(names, spans)}
            rows = []
            for eps in (1e-4, 1e-5, 1e-6):
                row = {"eps": eps}
                for prec, g in (("fp64", gf), ("bf16x3", gb)):
                    m.set_precision(prec)
                    v0, _ = m.evaluate(x)
                    v1, _ = m.evaluate(move(x, d, eps))
                    row[prec] = {"slope": (v1 - v0) / eps, "g_dot_d": float(g @ d)}
                rows.append(row)
            print(json.dumps({"mode": "slope_check", "config": args.fit_config, "logdet_probe": probe,
                              "objective_rel_err": abs(vb - vf) / abs(vf), "gradient_rel_l2_by_block": errs,
                              "slopes": rows}), flush=True)
    return 0


def fit_spread(args):
    """How far the fit's own discrete decisions carry rounding: the --fit-config fit to
    --fit-lbfgs steps from the seeded start and from starts whose X is scaled by (1 + eps z),
    z standard normal, in FP64 and in the precision form. One JSON line per fit."""
    import dataclasses

    import torch

    from gaspacho2_b200 import GPLVM, synth

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ds = synth.make(args.fit_config, 0, init=True)
    for prec, eps, seed in (("fp64", 0.0, 0), ("fp64", 1e-12, 1), ("fp64", 1e-12, 2), ("fp64", 1e-9, 3),
                            ("bf16x3", 0.0, 0), ("bf16x3", 1e-12, 1)):
        init = ds.init
        if eps:
            z = np.random.default_rng(seed).standard_normal(init.X.shape)
            init = dataclasses.replace(init, X=init.X * (1.0 + eps * z))
        with GPLVM.from_dataset(ds, stream=stream.cuda_stream, precision=prec) as m:
            m.set_params(init)
            m.kernel_mats()
            m.glm_init()
            rc, st, tr = m.fit(100000, args.fit_lbfgs)
        print(json.dumps({"config": args.fit_config, "lbfgs_budget": args.fit_lbfgs, "precision": prec, "eps": eps,
                          "seed": seed, "final_objective": float(tr[-1]), "outer_iterations": st["outer"],
                          "objective_evaluations": st["evals"], "nan_exit": bool(rc)}), flush=True)
    return 0


def precision_report(args):
    """The precision form against the plain FP64 path along a fit of --fit-config, every 10th
    L-BFGS step up to --fit-lbfgs: the two fits are run to each budget from the same seeded
    initialisation (the runs are deterministic, so the first k steps of a longer run are the
    k-step run), and compared on the objective, X and the GLM coefficients; at the precision
    fit's state both forms then evaluate the objective and gradient, which gives the
    per-evaluation errors along the trajectory. One JSON line per checkpoint."""
    import torch

    from gaspacho2_b200 import GPLVM, synth

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    torch.cuda.set_stream(stream)
    ds = synth.make(args.fit_config, 0, init=True)

    def fit(prec, budget):
        m = GPLVM.from_dataset(ds, stream=stream.cuda_stream, precision=prec)
        m.set_params(ds.init)
        torch.cuda.synchronize()
        t0 = time.time()
        m.kernel_mats()
        m.glm_init()
        rc, st, tr = m.fit(100000, budget)
        m.sync()
        return m, time.time() - t0, st, tr

    def rel(a, b):
        return float(np.linalg.norm(np.asarray(a) - np.asarray(b)) / max(np.linalg.norm(np.asarray(b)), 1e-300))

    for k in range(10, args.fit_lbfgs + 1, 10):
        mf, tf, sf, trf = fit("fp64", k)
        mb, tb, sb, trb = fit("bf16x3", k)
        row = {"config": args.fit_config, "lbfgs_steps": k, "seconds_fp64": tf, "seconds_bf16x3": tb,
               "objective_fp64": float(trf[-1]), "objective_bf16x3": float(trb[-1]),
               "objective_rel_diff": abs(trb[-1] - trf[-1]) / abs(trf[-1]),
               "X_rel_l2": rel(mb.get("X"), mf.get("X")), "beta_rel_l2": rel(mb.get("Beta"), mf.get("Beta")),
               "evals_fp64": sf["evals"], "evals_bf16x3": sb["evals"]}
        x = mb.params_vector()
        vb, gb = mb.evaluate(x)
        gb = gb.copy()
        mb.set_precision("fp64")
        vf, gf = mb.evaluate(x)
        row["at_bf16x3_state"] = {"objective_rel_err": abs(vb - vf) / abs(vf), "gradient_rel_l2": rel(gb, gf)}
        mf.close()
        mb.close()
        print(json.dumps(row), flush=True)
    return 0


def fit_trace(args):
    """The driver's fit of --fit-config, outer iteration by outer iteration (gpl_fit_outer), for
    each precision in --fit-precisions, under the --fit-lbfgs step budget: per outer iteration its
    IRLS sweeps, L-BFGS steps, objective evaluations, first and last accepted objective, why its
    L-BFGS phase ended and its device time; then the whole fit's time (CUDA events) and final
    objective. One JSON line per fit."""
    import torch

    from gaspacho2_b200 import GPLVM, synth

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    ds = synth.make(args.fit_config, 0, init=True)
    for prec in args.fit_precisions.split(","):
        with GPLVM.from_dataset(ds, stream=stream.cuda_stream, precision=prec) as m:
            if not args.plain:
                for k in ("fused_tail", "graph"):
                    m.set_option(k, 1)
            if args.eta_tc is not None:
                m.set_option("eta_tc", args.eta_tc)
            for kv in args.option:
                k, v = kv.split("=")
                m.set_option(k, int(v))
            m.set_params(ds.init)
            torch.cuda.synchronize()
            t0 = time.time()
            s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            s.record(stream)
            m.kernel_mats()
            m.glm_init()
            outer, left, itr = [], args.fit_lbfgs, 0
            while left > 0 and itr < args.fit_max_outer:
                a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                a.record(stream)
                rc, st, tr = m.fit_outer(itr, left)
                b.record(stream)
                torch.cuda.synchronize()
                left -= st["lbfgs"]
                d = np.abs(np.diff(tr)) / np.abs(tr[1:]) if len(tr) > 1 else np.zeros(0)
                why = "budget" if left <= 0 else ("stop test" if len(d) and d[-1] < 1e-8 else "step limit")
                outer.append({"itr": itr, "irls": st["irls"], "lbfgs": st["lbfgs"], "evals": st["evals"],
                              "first": float(tr[0]) if len(tr) else None, "last": float(tr[-1]) if len(tr) else None,
                              "ended": why, "seconds": a.elapsed_time(b) / 1e3,
                              "rejected_tries": int(st["evals"] - 1 - st["lbfgs"]),
                              "failed_line_searches": int(np.sum(np.diff(tr) <= 0)) if len(tr) > 1 else 0,
                              "rel_gains": [float(x) for x in (np.diff(tr) / np.abs(tr[1:]))[-5:]] if len(tr) > 1
                              else []})
                itr += 1
                if rc:
                    break
            e.record(stream)
            torch.cuda.synchronize()
            print(json.dumps({"mode": "fit_trace", "config": args.fit_config, "precision": prec,
                              "options": args.option, "ls_fp64_steps": m.get_option("ls_fp64_steps"),
                              "lbfgs_budget": args.fit_lbfgs, "seconds": s.elapsed_time(e) / 1e3,
                              "wall_seconds": time.time() - t0, "final_objective": outer[-1]["last"] if outer else None,
                              "outer": outer}), flush=True)
    return 0


def reference_gpu(args):
    """The reference's own CUDA build (oracle/_ref/ggplvm_gpu, the reference's sources compiled for
    sm_100a) beside this project's evaluation on the same seeded dataset of --config (use 0): the
    reference's median seconds per L-BFGS step of its first outer iteration (gradient, update and
    line-search objectives, from its printed trace), and this project's objective + gradient
    evaluation after its first IRLS phase, timed with CUDA events. One JSON line."""
    import torch

    from gaspacho2_b200 import GPLVM, synth
    from oracle import ref_gpu

    torch.cuda.set_device(0)
    kw = {}
    if args.N:
        kw["N"] = args.N
    if args.G:
        kw["G"] = args.G
    ds = synth.make(args.config, 0, init=True, **kw)
    line = {"mode": "reference_gpu", "config": workload_config(ds, args, "fp64")}
    if not ref_gpu.available():
        line["reference"] = {"unavailable": "oracle/_ref/ggplvm_gpu not built (make -C oracle ref-gpu)"}
    else:
        line["reference"] = ref_gpu.run(ds, steps=args.ref_gpu_steps, seconds=args.ref_gpu_seconds)
    stream = torch.cuda.Stream()
    with GPLVM.from_dataset(ds, stream=stream.cuda_stream) as m:
        for k in ("fused_tail", "graph"):
            m.set_option(k, 1)
        m.set_params(ds.init)
        m.kernel_mats()
        m.glm_init()
        m.irls(0, 200)
        m.objective_after_irls(0)
        for _ in range(3):
            m.evaluate_device()
        n = max(10, args.ref_gpu_steps)
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize()
        s.record(stream)
        for _ in range(n):
            m.evaluate_device()
        e.record(stream)
        torch.cuda.synchronize()
        t = s.elapsed_time(e) / 1e3 / n
        line["ours"] = {"seconds_per_evaluation": t, "evaluations_per_second": 1.0 / t,
                        "note": "objective + gradient after the first IRLS phase, CUDA-graph replay, CUDA events"}
    ref = line["reference"]
    if "seconds_per_lbfgs_step_median" in ref:
        line["reference_seconds_per_step_over_ours_per_evaluation"] = ref["seconds_per_lbfgs_step_median"] / t
    print(json.dumps(line), flush=True)
    return 0


def encoder_report(args):
    """The encoder's experiment (gaspacho2_b200.encoder.amortised_placement) alone: one JSON line per
    epoch count, each from a fresh fit of the training cells."""
    import torch

    from gaspacho2_b200.encoder import amortised_placement

    torch.cuda.set_device(0)
    stream = torch.cuda.Stream()
    epochs = [int(e) for e in args.enc_epochs_list.split(",") if e] or [args.enc_epochs]
    for ep in epochs:
        out = amortised_placement(args.enc_config, args.enc_train, args.enc_test, args.enc_fit_lbfgs, ep,
                                  n_genes=args.enc_genes, device=0, stream=stream.cuda_stream, lr=args.enc_lr)
        print(json.dumps({"mode": "encoder_report", **out}), flush=True)
    return 0


def main():
    args = parse()
    if args.encoder_report:
        return encoder_report(args)
    if args.slope_check:
        return slope_check(args)
    if args.reference_gpu:
        return reference_gpu(args)
    if args.fit_trace:
        return fit_trace(args)
    if args.precision_report:
        return precision_report(args)
    if args.fit_spread:
        return fit_spread(args)
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())

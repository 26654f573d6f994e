"""TEST INFRASTRUCTURE ONLY: runs the reference's own CUDA build (oracle/_ref/ggplvm_gpu, built by
`make -C oracle ref-gpu` from the reference's sources for sm_100a) on a seeded synthetic dataset
and times it, as the reference's GPU arm beside this project's kernels.

The reference's driver has no iteration budget (its outer loop runs to 5000 iterations,
ggplvm.cu:1146, its inner loops to 200/100 sweeps and 100 steps, :1152,1213) and no timer of its
own around a whole evaluation; it prints every objective value from the device ("lkhd[itr,jtr]=",
ggplvm.cu:812) and, after the L-BFGS update of every step, that kernel's time ("Update:", :1253).
This harness starts it with T and the other parameters from --init-params (the reference reads
them with readParams, util_cuda.cu:520-535), reads its output through a pseudo-terminal (so each
line arrives when printed; the driver synchronises the device after every launch) and stamps
each line with the host's monotonic clock. It stops the process once the L-BFGS phase of the
first outer iteration has taken `steps` steps or `seconds` have passed. The timed unit is one
L-BFGS step of that phase: the gradient (ggplvm.cu:1215-1240), the update and the line-search
objective evaluations (:1250-1289), from one step's "Update:" line to the next.
"""
from __future__ import annotations

import os
import pty
import re
import subprocess
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
BIN = os.path.join(HERE, "_ref", "ggplvm_gpu")


def _lines(f):
    """Lines of a pseudo-terminal until the other side closes it."""
    while True:
        try:
            line = f.readline()
        except OSError:  # EIO once the child has exited
            return
        if not line:
            return
        yield line


def available() -> bool:
    return os.path.exists(BIN)


def run(ds, steps: int = 20, seconds: float = 240.0, workdir: str | None = None) -> dict:
    """Times the reference's CUDA build on dataset `ds` (its init as --init-params)."""
    from gaspacho2_b200.formats import write_dataset

    wd = workdir or tempfile.mkdtemp(prefix="gpl_ref_gpu_")
    paths = write_dataset(wd, ds.y, ds.z, ds.ls, ds.X0, init=ds.init)
    cmd = [BIN, paths["Y"], paths["Z"], paths["ls"], paths["Xi"], "-M", str(ds.M), "-Q", str(ds.Q), "--init-params",
           paths["params"]]
    lk = re.compile(r"^lkhd\[(\d+),(\d+)\]=(\S+)")
    t0 = time.monotonic()
    master, slave = pty.openpty()
    proc = subprocess.Popen(cmd, cwd=wd, stdout=slave, stderr=slave, close_fds=True)
    os.close(slave)
    reader = os.fdopen(master, "r", errors="replace")
    step_t, lkhd_t, lkhd_v, lbfgs = [], [], [], False
    irls_lines = rejected = 0
    try:
        for line in _lines(reader):
            now = time.monotonic() - t0
            m = lk.match(line)
            if m:
                lkhd_t.append(now)
                lkhd_v.append(float(m.group(3)))
                if not lbfgs:
                    irls_lines += 1
            elif line.startswith("Update:"):
                lbfgs = True
                step_t.append(now)
            elif lbfgs and line.startswith("likelihood becomes lower"):
                rejected += 1
            if len(step_t) > steps or now > seconds:
                break
    finally:
        proc.kill()
        proc.wait()
        reader.close()
    elapsed = time.monotonic() - t0
    out = {"binary": "oracle/_ref/ggplvm_gpu", "N": ds.N, "G": ds.J, "M": ds.M, "Q": ds.Q,
           "wall_seconds": elapsed, "irls_objective_lines": irls_lines, "lbfgs_steps_seen": len(step_t),
           "rejected_tries": rejected}
    if len(step_t) >= 3:
        d = np.diff(np.array(step_t))
        # one step: the gradient, the update and its line-search objective evaluations
        out["seconds_per_lbfgs_step_median"] = float(np.median(d))
        out["seconds_per_lbfgs_step_mean"] = float(np.mean(d))
        out["objective_evaluations_in_steps"] = int(sum(1 for t in lkhd_t if step_t[0] < t <= step_t[-1]))
    out["last_objective"] = lkhd_v[-1] if lkhd_v else None
    return out

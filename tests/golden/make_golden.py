"""Generate the golden fixtures in this directory by running the reference.

Each case writes seeded inputs in the reference's restart format
(``G0.bin``, ``state0.bin``, ``job.config``), runs the reference driver
compiled from its own sources (``oracle/_ref/cosenu_ref_<variant>``, built by
``oracle/build.py``) through its ``--ff`` path, and stores what the reference
wrote: the ``rho_<t>.dat`` snapshots (16 significant digits), the
``survival_probability.dat`` and ``conserved_quantities.dat`` tables, and the
``time.txt`` loop time.  One case instead runs the reference's own
``initialize()`` (no ``--ff``) to pin the default initial condition.

Large cases keep a strided subset of the final state plus whole-state
checksums so that the files stay small.

Run:  python tests/golden/make_golden.py [case ...]
"""
from __future__ import annotations

import hashlib
import json
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)

from oracle.build import build, ref_binary  # noqa: E402
from oracle.oracle import (Case, Oracle, read_rho_dat, read_table, run_reference,  # noqa: E402
                           write_job_config, job_config_dict, interior)

SEED = 20240601

# name -> (Case kwargs, n_iter, anal_every, n_dump_rho, big)
# Small grids use a box with dz = 1 (dt = 0.4): on [-600, 600] a 64-cell grid
# has dt = 7.5 and mu*dt far outside RK4's stability region (the reference
# itself then produces NaN).
SB = dict(z0=-32.0, z1=32.0)
CASES = {
    # the small FV workload's physics (omega = 0, mu = 1) on a small grid
    "fv_small": (dict(nz=64, nvz=16, gz=4, scheme="fv", omega=0.0, **SB), 21, 5, 4, False),
    # FV with a vacuum term (cosenu_configs.yaml defaults: omega 1e-2, theta 37 deg)
    "fv_vac": (dict(nz=64, nvz=16, gz=4, scheme="fv", omega=1e-2, theta_deg=37.0, **SB), 21, 5, 4, False),
    # odd nvz puts a v = 0 row on the grid (sign(v) = 0 branch of rhs_fv.hpp:147-162)
    "fv_oddv": (dict(nz=32, nvz=15, gz=4, scheme="fv", omega=1e-2, theta_deg=37.0, z0=-16.0,
                      z1=16.0), 11, 5, 2, False),
    # the large FD workload's physics (omega 1e-3, theta 1e-6 deg, NO) on a small grid
    "fd_small": (dict(nz=64, nvz=16, gz=2, scheme="fd", omega=1e-3, theta_deg=1e-6, **SB), 21, 5, 4, False),
    "fd_vac": (dict(nz=64, nvz=16, gz=2, scheme="fd", omega=1e-2, theta_deg=37.0, pmo=-1.0, **SB),
               21, 5, 4, False),
    "fv_open": (dict(nz=64, nvz=16, gz=4, scheme="fv", bc="open", omega=1e-2, theta_deg=37.0, **SB),
                11, 5, 2, False),
    "fd_open": (dict(nz=64, nvz=16, gz=2, scheme="fd", bc="open", omega=1e-2, theta_deg=37.0, **SB),
                11, 5, 2, False),
    "fv_mat": (dict(nz=64, nvz=16, gz=4, scheme="fv", mat=True, omega=1e-2, theta_deg=37.0, **SB),
               11, 5, 2, False),
    "fd_mat": (dict(nz=64, nvz=16, gz=2, scheme="fd", mat=True, omega=1e-2, theta_deg=37.0, **SB),
               11, 5, 2, False),
    "fd_ko5": (dict(nz=64, nvz=16, gz=3, scheme="fd", ko_order=5, omega=1e-2, theta_deg=37.0, **SB),
               11, 5, 2, False),
    "fv_advoff": (dict(nz=64, nvz=16, gz=4, scheme="fv", advec_off=True, omega=1e-2,
                       theta_deg=37.0, **SB), 11, 5, 2, False),
    "fd_advoff": (dict(nz=64, nvz=16, gz=2, scheme="fd", advec_off=True, omega=1e-2,
                       theta_deg=37.0, **SB), 11, 5, 2, False),
    # the small FV workload exactly: nz 1024, nvz 64, 500 steps (pre-saturation)
    "c1_pre": (dict(nz=1024, nvz=64, gz=4, scheme="fv", omega=0.0), 501, 50, 2, True),
    # the 1024 x 64 FV grid run through saturation (<Pee> leaves 1 near step 350)
    "c1_sat": (dict(nz=1024, nvz=64, gz=4, scheme="fv", omega=0.0), 1501, 25, 3, True),
}

SUBSET_STRIDE = 16  # z stride of the stored subset for big cases
TEXT_PIN_CASES = ("fv_small", "fd_small")

# Full-size grids of the large workloads, truncated to a few steps (the reference
# needs N_ITER >= 10, src/main.cpp:195).  Each stores a column subset of the
# dumped state (every v row and component at a few z columns: both periodic
# edges and seeded random columns), per-row checksums of the whole state and the
# analysis rows.
#   name -> (Case kwargs, n_iter, anal_every, n_dump_rho, subset columns)
FULL_CASES = {
    # FD (central FD4 + KO3) at nz 32768 x nvz 256: dumps at steps 5 and 10
    "c2_ref": (dict(nz=32768, nvz=256, gz=2, z0=-3000.0, z1=3000.0, scheme="fd", pmo=1.0,
                    omega=1e-3, theta_deg=1e-6, mu=1.0), 11, 5, 2, 32),
    # FV (WENO7) at nz 65536 x nvz 512: analysis at steps 3, 6, 9, dump at step 5
    "c3_ref": (dict(nz=65536, nvz=512, gz=4, scheme="fv", omega=0.0, mu=1.0), 10, 3, 2, 16),
}


def subset_columns(nz: int, ncol: int) -> np.ndarray:
    """Both periodic edges (4 columns each) plus seeded random interior columns."""
    rng = np.random.default_rng(nz)
    edge = np.concatenate([np.arange(4), np.arange(nz - 4, nz)])
    rest = np.setdiff1d(np.arange(nz), edge)
    return np.sort(np.concatenate([edge, rng.choice(rest, ncol - 8, replace=False)]))


def row_checksums(s: np.ndarray) -> np.ndarray:
    """Per component and v row: sum, sum of squares and sum of |x| over z."""
    return np.stack([s.sum(axis=2), (s * s).sum(axis=2), np.abs(s).sum(axis=2)], -1)


def read_rho_dat_fast(path: str, case: Case) -> np.ndarray:
    """rho_<t>.dat of a large grid -> [8][nvz][nz] (pandas' C tokenizer; the
    text has z blocks of nvz lines of 10 numbers)."""
    import pandas as pd
    a = pd.read_csv(path, sep=r"\s+", header=None, dtype=np.float64, engine="c",
                    skip_blank_lines=True).to_numpy()
    a = a.reshape(case.nz, case.nvz, 10)
    return np.ascontiguousarray(np.transpose(a[:, :, 2:], (2, 1, 0)))


def make_full_case(name: str, o: Oracle) -> None:
    import shutil
    kw, n_iter, anal, ndump, ncol = FULL_CASES[name]
    case = Case(**kw)
    G, bG, st0 = o.init_seeded(case, seed=SEED)
    wd = tempfile.mkdtemp(prefix=f"cosenu_{name}_")
    try:
        r = run_reference(case, G, bG, st0, n_iter=n_iter, anal_every=anal, n_dump_rho=ndump,
                          workdir=wd, nthreads=os.cpu_count() or 1, timeout=6 * 3600,
                          read_dumps=False)
        files = r["files"]
        dumps = sorted(int(f[4:-4]) for f in os.listdir(wd) if f.startswith("rho_"))
        cols = subset_columns(case.nz, ncol)
        s0 = interior(case, st0)
        out = {"case": json.dumps(kw), "seed": SEED, "n_iter": n_iter, "anal_every": anal,
               "n_dump_rho": ndump, "dump_steps": np.array(dumps, dtype=np.int64),
               "columns": cols,
               "survival_probability": read_table_text(files["survival_probability.dat"]),
               "conserved_quantities": read_table_text(files["conserved_quantities.dat"]),
               "ref_loop_seconds": r["loop_seconds"], "ref_threads": os.cpu_count() or 1,
               "state0_sha256": hashlib.sha256(s0.tobytes()).hexdigest()}
        for t in dumps:
            s = read_rho_dat_fast(os.path.join(wd, f"rho_{t}.dat"), case)
            if not np.all(np.isfinite(s)):
                raise RuntimeError(f"{name}: reference output at step {t} is not finite")
            out[f"rho_{t}_columns"] = np.ascontiguousarray(s[:, :, cols])
            out[f"rho_{t}_row_checksums"] = row_checksums(s)
            out[f"rho_{t}_pee_v"] = s[0].sum(axis=1) / s0[0].sum(axis=1)
            out[f"rho_{t}_pbee_v"] = s[4].sum(axis=1) / s0[4].sum(axis=1)
            del s
    finally:
        shutil.rmtree(wd, ignore_errors=True)
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: dumps {dumps}, loop {r['loop_seconds']:.1f}s")


def _b(txt: str) -> np.ndarray:
    """Text stored as raw bytes (uint8) inside the npz."""
    return np.frombuffer(txt.encode(), dtype=np.uint8)


def state_checksums(s: np.ndarray) -> np.ndarray:
    """Per component: sum, sum of squares, sum of |x| (interior)."""
    return np.stack([s.sum(axis=(1, 2)), (s * s).sum(axis=(1, 2)), np.abs(s).sum(axis=(1, 2))], 1)


def make_case(name: str, o: Oracle) -> None:
    kw, n_iter, anal, ndump, big = CASES[name]
    case = Case(**kw)
    G, bG, st0 = o.init_seeded(case, seed=SEED)
    r = run_reference(case, G, bG, st0, n_iter=n_iter, anal_every=anal, n_dump_rho=ndump,
                      nthreads=os.cpu_count() or 1)
    files = r["files"]
    dumps = sorted(int(f[4:-4]) for f in files if f.startswith("rho_"))
    out = {"case": json.dumps(kw), "seed": SEED, "n_iter": n_iter, "anal_every": anal,
           "n_dump_rho": ndump, "dump_steps": np.array(dumps, dtype=np.int64),
           "survival_probability": read_table_text(files["survival_probability.dat"]),
           "conserved_quantities": read_table_text(files["conserved_quantities.dat"]),
           "survival_probability_txt": _b(files["survival_probability.dat"]),
           "conserved_quantities_txt": _b(files["conserved_quantities.dat"]),
           "ref_loop_seconds": r["loop_seconds"],
           "state0_sha256": hashlib.sha256(interior(case, st0).tobytes()).hexdigest()}
    with tempfile.TemporaryDirectory() as d:
        for t in dumps:
            p = os.path.join(d, "rho.dat")
            open(p, "w").write(files[f"rho_{t}.dat"])
            s = read_rho_dat(p, case)
            if not np.all(np.isfinite(s)):
                raise RuntimeError(f"{name}: reference output at step {t} is not finite")
            if big:
                out[f"rho_{t}_subset"] = np.ascontiguousarray(s[:, :, ::SUBSET_STRIDE])
                out[f"rho_{t}_checksums"] = state_checksums(s)
                out[f"rho_{t}_pee_v"] = s[0].sum(axis=1) / interior(case, st0)[0].sum(axis=1)
                out[f"rho_{t}_pbee_v"] = s[4].sum(axis=1) / interior(case, st0)[4].sum(axis=1)
            else:
                out[f"rho_{t}"] = s
    if not big:
        out["G"] = interior(case, G).copy()
        out["bG"] = interior(case, bG).copy()
        out["state0"] = interior(case, st0).copy()
    if name in TEXT_PIN_CASES:
        # the first dump file verbatim, to pin the text format byte for byte
        out["rho_first_txt"] = _b(files[f"rho_{dumps[0]}.dat"])
    np.savez_compressed(os.path.join(HERE, f"{name}.npz"), **out)
    print(f"{name}: dumps {dumps}, loop {r['loop_seconds']:.3f}s")


def make_default_ic(o: Oracle) -> None:
    """Reference initialize() path (fresh start, no --ff): pins the default
    initial condition (src/initialize.hpp) and the t = 0 analysis rows."""
    kw = dict(nz=64, nvz=16, gz=4, scheme="fv", omega=1e-2, theta_deg=37.0, **SB)
    case = Case(**kw)
    pert = 1e-3
    with tempfile.TemporaryDirectory() as d:
        write_job_config(os.path.join(d, "job.config"),
                         job_config_dict(case, 11, 5, 2, perturbation_size=pert))
        env = dict(os.environ, OMP_NUM_THREADS="2")
        subprocess.run([ref_binary("fv"), "--conf", "job.config"], cwd=d, env=env, check=True,
                       capture_output=True)
        g0 = np.fromfile(os.path.join(d, "G0.bin"), "<f8").reshape(case.nvz, case.nz, 2)
        s0 = np.fromfile(os.path.join(d, "state0.bin"), "<f8").reshape(case.nvz, case.nz, 8)
        files = {f: open(os.path.join(d, f)).read() for f in os.listdir(d) if f.endswith(".dat")}
        rho0 = read_rho_dat(os.path.join(d, "rho_0.dat"), case)
        rho10 = read_rho_dat(os.path.join(d, "rho_10.dat"), case)
    np.savez_compressed(os.path.join(HERE, "fv_default_ic.npz"), case=json.dumps(kw),
                        perturbation_size=pert, G0=g0, state0=s0, rho_0=rho0, rho_10=rho10,
                        rho_0_txt=_b(files["rho_0.dat"]),
                        survival_probability_txt=_b(files["survival_probability.dat"]),
                        conserved_quantities_txt=_b(files["conserved_quantities.dat"]))
    print("fv_default_ic: done")


def read_table_text(txt: str) -> np.ndarray:
    rows = [ln.split() for ln in txt.splitlines() if ln.strip() and not ln.startswith("#")]
    return np.array(rows, dtype=np.float64)


def main(argv: list[str]) -> None:
    build()
    o = Oracle()
    names = argv or list(CASES) + ["fv_default_ic"] + list(FULL_CASES)
    for n in names:
        if n == "fv_default_ic":
            make_default_ic(o)
        elif n in FULL_CASES:
            make_full_case(n, o)
        else:
            make_case(n, o)


if __name__ == "__main__":
    main(sys.argv[1:])

"""Python handle on the oracle (test infrastructure only).

* ``Oracle`` -- ctypes wrapper of ``libcosenu_oracle.so`` (the C restatement
  in ``cosenu_oracle.c``), working on numpy arrays in the reference layout
  ``[8][nvz][nz+2gz]`` (src/nuosc.hpp:145-148 of COSEnu).
* Readers and writers for the reference's files: ``job.config``
  (manage.py:116-121 ``write_dict``), ``G0.bin`` / ``state0.bin``
  (src/snaps.hpp:41-183), ``rho_<t>.dat`` (src/snaps.hpp:187-218),
  ``survival_probability.dat`` / ``conserved_quantities.dat``
  (src/analysis.hpp:71-185).
* ``run_reference`` -- runs a reference binary from ``oracle/_ref`` on such
  inputs through its own ``--ff`` restart path (src/main.cpp:144-151).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg import
this module.
"""
from __future__ import annotations

import ctypes as C
import dataclasses
import os
import subprocess
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
NCOMP = 8
COMPONENTS = ("ee", "xx", "ex_re", "ex_im", "bee", "bxx", "bex_re", "bex_im")
DIAG_SLOTS = ("dP_max", "avdP", "avbdP", "M0", "M0_e1", "M0_e2", "M0_e3", "Pee", "Pbee",
              "trace", "btrace", "eln")


class _CParams(C.Structure):
    _fields_ = [("nz", C.c_int), ("nvz", C.c_int), ("gz", C.c_int),
                ("z0", C.c_double), ("z1", C.c_double), ("v0", C.c_double), ("v1", C.c_double),
                ("cfl", C.c_double), ("pmo", C.c_double), ("omega", C.c_double),
                ("theta_deg", C.c_double), ("mu", C.c_double),
                ("scheme", C.c_int), ("bc", C.c_int), ("vac", C.c_int), ("mat", C.c_int),
                ("coll", C.c_int), ("advec_off", C.c_int), ("fd_advec", C.c_int),
                ("ko_order", C.c_int), ("coll_direct", C.c_int), ("nthreads", C.c_int)]


@dataclasses.dataclass
class Case:
    """One simulation set-up; fields mirror the job.config keys plus the
    compile-time switches of src/presets.hpp."""
    nz: int = 64
    nvz: int = 16
    gz: int = 4
    z0: float = -600.0
    z1: float = 600.0
    v0: float = -1.0
    v1: float = 1.0
    cfl: float = 0.4
    pmo: float = 1.0
    omega: float = 0.0
    theta_deg: float = 0.0
    mu: float = 1.0
    scheme: str = "fv"          # "fv" | "fd"
    bc: str = "periodic"        # "periodic" | "open"
    vac: bool = True
    mat: bool = False
    coll: bool = True
    advec_off: bool = False
    fd_advec: str = "center"    # "center" | "upwind" | "lopsided"
    ko_order: int = 3

    @property
    def ld(self) -> int:
        return self.nz + 2 * self.gz

    @property
    def dz(self) -> float:
        return (self.z1 - self.z0) / self.nz

    @property
    def dv(self) -> float:
        return (self.v1 - self.v0) / self.nvz

    @property
    def dt(self) -> float:
        return self.cfl * self.dz

    def ref_variant(self) -> str:
        """Name of the oracle/_ref binary compiled with matching switches."""
        v = self.scheme
        if self.bc == "open":
            v += "_open"
        if self.mat:
            v += "_mat"
        if self.scheme == "fd" and self.ko_order == 5:
            v += "_ko5"
        if self.advec_off:
            v += "_advoff"
        if not (self.vac and self.coll) or (self.scheme == "fd" and self.fd_advec != "center"):
            raise ValueError("no reference build for this switch combination")
        return v

    def cparams(self, coll_direct: bool = False, nthreads: int = 0) -> _CParams:
        return _CParams(self.nz, self.nvz, self.gz, self.z0, self.z1, self.v0, self.v1, self.cfl,
                        self.pmo, self.omega, self.theta_deg, self.mu,
                        0 if self.scheme == "fv" else 1, 0 if self.bc == "periodic" else 1,
                        int(self.vac), int(self.mat), int(self.coll), int(self.advec_off),
                        {"center": 0, "upwind": 1, "lopsided": 2}[self.fd_advec], self.ko_order,
                        int(coll_direct), nthreads)


_P = np.ctypeslib.ndpointer(dtype=np.float64, flags="C_CONTIGUOUS")


class Oracle:
    def __init__(self, so_path: str | None = None):
        if so_path is None:
            from oracle.build import build_oracle
            so_path = build_oracle()
        lib = C.CDLL(so_path)
        pp = C.POINTER(_CParams)
        lib.orc_step_rk4.argtypes = [pp, _P, C.c_int]
        lib.orc_step_rk4.restype = C.c_int
        lib.orc_rhs.argtypes = [pp, _P, _P]
        lib.orc_weno7.argtypes = [pp, _P, _P, _P]
        lib.orc_fill_ghosts.argtypes = [pp, _P, C.c_int]
        lib.orc_grid_info.argtypes = [pp, _P, _P, _P]
        lib.orc_init_seeded.argtypes = [pp, C.c_uint64, C.c_uint32, C.c_double, C.c_double,
                                        C.c_double, C.c_double, _P, _P, _P]
        lib.orc_init_reference.argtypes = [pp, C.c_double, _P, _P, _P]
        lib.orc_analyse.argtypes = [pp, _P, _P, _P, _P, _P]
        lib.orc_pee_v.argtypes = [pp, _P, _P, _P, _P]
        lib.orc_philox.argtypes = [C.c_uint32] * 6 + [np.ctypeslib.ndpointer(np.uint32)]
        self.lib = lib

    # -- state helpers -------------------------------------------------------
    @staticmethod
    def empty_state(case: Case) -> np.ndarray:
        return np.zeros((NCOMP, case.nvz, case.ld), dtype=np.float64)

    def grid(self, case: Case):
        Z = np.zeros(case.nz)
        vz = np.zeros(case.nvz)
        s = np.zeros(5)
        self.lib.orc_grid_info(C.byref(case.cparams()), Z, vz, s)
        return Z, vz, dict(zip(("dz", "dv", "dt", "ct", "st"), s))

    def init_seeded(self, case: Case, seed: int = 1234, instance: int = 0, sig_nu: float = 0.6,
                    sig_nubar: float = 0.5, alpha: float = 0.9, amp: float = 1e-6):
        G = np.zeros((case.nvz, case.ld))
        bG = np.zeros((case.nvz, case.ld))
        st = self.empty_state(case)
        self.lib.orc_init_seeded(C.byref(case.cparams()), seed, instance, sig_nu, sig_nubar, alpha,
                                 amp, G, bG, st)
        return G, bG, st

    def init_reference(self, case: Case, perturbation_size: float = 0.0):
        G = np.zeros((case.nvz, case.ld))
        bG = np.zeros((case.nvz, case.ld))
        st = self.empty_state(case)
        self.lib.orc_init_reference(C.byref(case.cparams()), perturbation_size, G, bG, st)
        return G, bG, st

    def fill_ghosts(self, case: Case, f: np.ndarray) -> np.ndarray:
        f = np.ascontiguousarray(f, dtype=np.float64).copy()
        n = f.size // (case.nvz * case.ld)
        self.lib.orc_fill_ghosts(C.byref(case.cparams()), f, n)
        return f

    def step(self, case: Case, state: np.ndarray, nsteps: int, coll_direct: bool = False,
             nthreads: int = 0) -> np.ndarray:
        y = np.ascontiguousarray(state, dtype=np.float64).copy()
        rc = self.lib.orc_step_rk4(C.byref(case.cparams(coll_direct, nthreads)), y, nsteps)
        if rc != 0:
            raise MemoryError("oracle step failed")
        return y

    def rhs(self, case: Case, state: np.ndarray, coll_direct: bool = False) -> np.ndarray:
        x = self.fill_ghosts(case, state)
        out = self.empty_state(case)
        self.lib.orc_rhs(C.byref(case.cparams(coll_direct)), out, x)
        return out

    def weno7(self, case: Case, comp: np.ndarray):
        r = np.zeros((case.nvz, case.ld))
        l = np.zeros((case.nvz, case.ld))
        self.lib.orc_weno7(C.byref(case.cparams()), np.ascontiguousarray(comp), r, l)
        return r, l

    def analyse(self, case: Case, state, G, bG, state0) -> dict:
        out = np.zeros(len(DIAG_SLOTS))
        self.lib.orc_analyse(C.byref(case.cparams()), np.ascontiguousarray(state),
                             np.ascontiguousarray(G), np.ascontiguousarray(bG),
                             np.ascontiguousarray(state0), out)
        return dict(zip(DIAG_SLOTS, out.tolist()))

    def pee_v(self, case: Case, state, state0):
        a = np.zeros(case.nvz)
        b = np.zeros(case.nvz)
        self.lib.orc_pee_v(C.byref(case.cparams()), np.ascontiguousarray(state),
                           np.ascontiguousarray(state0), a, b)
        return a, b

    def philox(self, ctr, key) -> np.ndarray:
        out = np.zeros(4, dtype=np.uint32)
        self.lib.orc_philox(*[int(c) for c in ctr], int(key[0]), int(key[1]), out)
        return out


def interior(case: Case, f: np.ndarray) -> np.ndarray:
    return f[..., case.gz:case.gz + case.nz]


# -- reference file formats ---------------------------------------------------

def job_config_dict(case: Case, n_iter: int, anal_every: int, n_dump_rho: int,
                    perturbation_size: float = 0.0) -> dict:
    """The job.config keys manage.py:236-256 writes (dz/dt are informational;
    the binary recomputes them, src/nuosc.hpp:78-80)."""
    return {"scheme": case.scheme.upper(), "z0": case.z0, "z1": case.z1, "nvz": case.nvz,
            "CFL": case.cfl, "dz": case.dz, "dt": case.dt, "gz": case.gz, "v0": case.v0,
            "v1": case.v1, "nz": case.nz, "pmo": case.pmo, "omega": case.omega,
            "theta": case.theta_deg, "mu": case.mu, "perturbation_size": perturbation_size,
            "N_ITER": n_iter, "ANAL_EVERY": anal_every, "n_dump_rho": n_dump_rho}


def write_job_config(path: str, d: dict) -> None:
    """Same layout as manage.py's write_dict (manage.py:116-121)."""
    m = max(len(k) for k in d)
    with open(path, "w") as f:
        for k, v in d.items():
            f.write(f"{str(k).ljust(m + 1)} : {v!r} \n" if isinstance(v, float)
                    else f"{str(k).ljust(m + 1)} : {v} \n")


def write_G0_bin(path: str, case: Case, G: np.ndarray, bG: np.ndarray) -> None:
    """Interleaved (G, bG) per interior cell, v-major (src/snaps.hpp:160-183)."""
    a = np.stack([interior(case, G), interior(case, bG)], axis=-1)
    a.astype("<f8").tofile(path)


def write_state_bin(path: str, case: Case, state: np.ndarray, t: int | None = None) -> None:
    """8 interleaved doubles per interior cell, v-major; ``state.bin`` carries
    an int32 iteration first, ``state0.bin`` does not (src/snaps.hpp:6-71)."""
    a = np.moveaxis(interior(case, state), 0, -1).astype("<f8")
    with open(path, "wb") as f:
        if t is not None:
            f.write(np.int32(t).tobytes())
        f.write(a.tobytes())


def read_state_bin(path: str, case: Case, header: bool) -> tuple[np.ndarray, int | None]:
    raw = open(path, "rb").read()
    t = None
    if header:
        t = int(np.frombuffer(raw[:4], "<i4")[0])
        raw = raw[4:]
    a = np.frombuffer(raw, "<f8").reshape(case.nvz, case.nz, NCOMP)
    st = np.zeros((NCOMP, case.nvz, case.ld))
    st[..., case.gz:case.gz + case.nz] = np.moveaxis(a, -1, 0)
    return st, t


def read_rho_dat(path: str, case: Case) -> np.ndarray:
    """rho_<t>.dat -> interior state [8][nvz][nz] (src/snaps.hpp:201-214:
    z outer, v inner, blank line after each z block)."""
    rows = [ln.split() for ln in open(path) if ln.strip()]
    a = np.array(rows, dtype=np.float64).reshape(case.nz, case.nvz, 10)
    return np.ascontiguousarray(np.transpose(a[:, :, 2:], (2, 1, 0)))


def read_table(path: str) -> np.ndarray:
    rows = [ln.split() for ln in open(path) if ln.strip() and not ln.startswith("#")]
    return np.array(rows, dtype=np.float64)


# -- running the reference ---------------------------------------------------

def run_reference(case: Case, G, bG, state0, n_iter: int, anal_every: int, n_dump_rho: int,
                  workdir: str | None = None, nthreads: int = 0, exe: str | None = None,
                  timeout: float = 3600, read_dumps: bool = True) -> dict:
    """Run the reference binary through its --ff path; returns the files it
    wrote (text; the rho_<t>.dat snapshots only with ``read_dumps``, they stay
    in ``workdir`` otherwise) and the parsed loop time (time.txt)."""
    from oracle.build import ref_binary
    exe = exe or ref_binary(case.ref_variant())
    if not os.path.exists(exe):
        raise FileNotFoundError(exe)
    own = workdir is None
    wd = workdir or tempfile.mkdtemp(prefix="cosenu_ref_")
    write_job_config(os.path.join(wd, "job.config"),
                     job_config_dict(case, n_iter, anal_every, n_dump_rho))
    write_G0_bin(os.path.join(wd, "G0.bin"), case, G, bG)
    write_state_bin(os.path.join(wd, "state0.bin"), case, state0)
    env = dict(os.environ)
    env["OMP_NUM_THREADS"] = str(nthreads or os.cpu_count() or 1)
    p = subprocess.run([exe, "--conf", "job.config", "--ff"], cwd=wd, env=env,
                       capture_output=True, text=True, timeout=timeout)
    if p.returncode != 0:
        raise RuntimeError(f"reference exited {p.returncode}: {p.stdout[-400:]} {p.stderr[-400:]}")
    files = {}
    for fn in os.listdir(wd):
        if fn.startswith("rho_") and not read_dumps:
            continue
        if fn.endswith(".dat") or fn == "time.txt":
            files[fn] = open(os.path.join(wd, fn)).read()
    out = {"files": files, "workdir": wd, "stdout": p.stdout,
           "loop_seconds": float(files["time.txt"].split()[0])}
    if own and os.environ.get("COSENU_KEEP_REF_DIR") is None:
        import shutil
        out["workdir"] = None
        shutil.rmtree(wd, ignore_errors=True)
    return out

"""Python face of the B200 path, shaped like the reference's NuOsc class
(src/nuosc.hpp:7-191 of COSEnu): construct from the job.config parameters,
load or initialise a state, call ``step_rk4()`` (or ``evolve(n)``), analyse.

State arrays use the reference layout ``[8][nvz][nz + 2*gz]`` (component
order ee, xx, ex_re, ex_im, bee, bxx, bex_re, bex_im).  Everything runs in
the CUDA library; there is no CPU path.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib as L

COMPONENTS = ("ee", "xx", "ex_re", "ex_im", "bee", "bxx", "bex_re", "bex_im")
_SCHEMES = {"fv": L.FV, "fd": L.FD}
_BCS = {"periodic": L.PERIODIC, "open": L.OPEN}
_FDADV = {"center": L.FD_CENTER, "upwind": L.FD_UPWIND, "lopsided": L.FD_LOPSIDED}
_PREC = {"fp64": L.FP64, "fp32": L.FP32_BULK, "fp32_bulk": L.FP32_BULK}


def make_params(nz: int, nvz: int, gz: int = 4, z0: float = -600.0, z1: float = 600.0,
                v0: float = -1.0, v1: float = 1.0, cfl: float = 0.4, pmo: float = 1.0,
                omega: float = 0.0, theta_deg: float = 0.0, mu: float = 1.0,
                scheme: str = "fv", bc: str = "periodic", vac: bool = True, mat: bool = False,
                coll: bool = True, advec_off: bool = False, fd_advec: str = "center",
                ko_order: int = 3, precision: str = "fp64", device: int = 0, tile_z: int = 0,
                tile_v: int = 0) -> L.Params:
    p = L.Params()
    p.nz, p.nvz, p.gz = nz, nvz, gz
    p.z0, p.z1, p.v0, p.v1, p.cfl = z0, z1, v0, v1, cfl
    p.pmo, p.omega, p.theta_deg, p.mu = pmo, omega, theta_deg, mu
    p.scheme = _SCHEMES[scheme]
    p.bc = _BCS[bc]
    p.flags = (L.VAC if vac else 0) | (L.MAT if mat else 0) | (L.COLL if coll else 0) | \
        (L.ADVEC_OFF if advec_off else 0)
    p.fd_advec = _FDADV[fd_advec]
    p.ko_order = ko_order
    p.precision = _PREC[precision]
    p.device = device
    p.tile_z, p.tile_v = tile_z, tile_v
    return p


def _ptrs(arr: np.ndarray) -> "L.DPTR8":
    return L.DPTR8(*[arr[c].ctypes.data for c in range(8)])


class NuOsc:
    """One simulation held on one GPU."""

    def __init__(self, params: L.Params | None = None, **kw):
        self.lib = L.load()
        self.p = params if params is not None else make_params(**kw)
        h = C.c_void_p()
        rc = self.lib.cosenu_create(C.byref(self.p), C.byref(h))
        if rc != L.OK:
            raise L.CosenuError(rc, self.lib.cosenu_last_error(None).decode())
        self.h = h
        self._owned = True
        self._init_grid()

    @classmethod
    def _member(cls, handle: int, params: L.Params) -> "NuOsc":
        """View of an ensemble member (the ensemble owns the context)."""
        self = cls.__new__(cls)
        self.lib = L.load()
        self.p = params
        self.h = C.c_void_p(handle)
        self._owned = False
        self._init_grid()
        return self

    def _init_grid(self):
        g = (C.c_double * 5)()
        self.lib.cosenu_grid(self.h, g)
        self.dz, self.dv, self.dt, self.ct, self.st = list(g)
        self.nz, self.nvz, self.gz = self.p.nz, self.p.nvz, self.p.gz

    # -- plumbing -------------------------------------------------------------
    def _check(self, rc: int) -> None:
        if rc != L.OK:
            raise L.CosenuError(rc, self.lib.cosenu_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            if getattr(self, "_owned", True):
                self.lib.cosenu_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    @property
    def ld(self) -> int:
        return self.nz + 2 * self.gz

    def empty_state(self) -> np.ndarray:
        return np.zeros((8, self.nvz, self.ld), dtype=np.float64)

    def _host(self, a: np.ndarray, planes: int) -> np.ndarray:
        a = np.ascontiguousarray(a, dtype=np.float64)
        if a.shape != ((planes,) if planes > 1 else ()) + (self.nvz, self.ld):
            raise ValueError(f"expected shape {(planes, self.nvz, self.ld)}, got {a.shape}")
        return a

    def set_stream(self, stream_handle: int | None) -> None:
        self._check(self.lib.cosenu_set_stream(self.h, stream_handle))

    # -- NuOsc-shaped API -------------------------------------------------------
    def set_vac_pars(self, pmo: float, omega: float, theta_deg: float) -> None:
        self._check(self.lib.cosenu_set_vac_pars(self.h, pmo, omega, theta_deg))
        g = (C.c_double * 5)()
        self.lib.cosenu_grid(self.h, g)
        self.ct, self.st = g[3], g[4]

    def set_collective_pars(self, mu: float) -> None:
        self._check(self.lib.cosenu_set_collective_pars(self.h, mu))

    def upload(self, state: np.ndarray) -> None:
        s = self._host(state, 8)
        self._check(self.lib.cosenu_upload(self.h, _ptrs(s), self.gz))

    def download(self) -> np.ndarray:
        out = self.empty_state()
        self._check(self.lib.cosenu_download(self.h, _ptrs(out), self.gz))
        return out

    v_stat = property(download)

    def snapshot(self) -> int:
        """Starts an asynchronous copy of the current state to pinned host
        memory (cosenu_snapshot); returns the step count it was taken at."""
        n = C.c_longlong()
        self._check(self.lib.cosenu_snapshot(self.h, C.byref(n)))
        return n.value

    def snapshot_wait(self) -> np.ndarray:
        """Waits for the last snapshot and returns a copy of it as [8][nvz][nz]
        (interior cells)."""
        p = C.POINTER(C.c_double)()
        self._check(self.lib.cosenu_snapshot_wait(self.h, C.byref(p)))
        n = 8 * self.nvz * self.nz
        return np.ctypeslib.as_array(p, shape=(n,)).reshape(8, self.nvz, self.nz).copy()

    def set_profile(self, G: np.ndarray, bG: np.ndarray) -> None:
        G = self._host(G, 1)
        bG = self._host(bG, 1)
        self._check(self.lib.cosenu_set_profile(self.h, G.ctypes.data, bG.ctypes.data, self.gz))

    def set_state0(self, state0: np.ndarray) -> None:
        s = self._host(state0, 8)
        self._check(self.lib.cosenu_set_state0(self.h, _ptrs(s), self.gz))

    def mark_state0(self) -> None:
        self._check(self.lib.cosenu_mark_state0(self.h))

    def initialize(self, perturbation_size: float = 0.0) -> None:
        """NuOsc::initialize (src/initialize.hpp:6-47), on the device."""
        self._check(self.lib.cosenu_init_reference(self.h, perturbation_size))

    def init_seeded(self, seed: int, instance: int = 0, sig_nu: float = 0.6,
                    sig_nubar: float = 0.5, alpha: float = 0.9, amp: float = 1e-6) -> None:
        self._check(self.lib.cosenu_init_seeded(self.h, seed, instance, sig_nu, sig_nubar, alpha,
                                                amp))

    def step_rk4(self) -> None:
        self._check(self.lib.cosenu_step(self.h, 1))

    def evolve(self, nsteps: int) -> None:
        self._check(self.lib.cosenu_step(self.h, nsteps))

    def step_stage(self, stage: int) -> None:
        self._check(self.lib.cosenu_step_stage(self.h, stage))

    def prepare_graphs(self) -> None:
        """Capture the CUDA graphs of evolve() now rather than on first use."""
        self._check(self.lib.cosenu_prepare_graphs(self.h))

    def synchronize(self) -> None:
        self._check(self.lib.cosenu_synchronize(self.h))

    def set_wait_limit(self, seconds: float) -> None:
        """Time limit of each pipeline wait inside the TMA stage kernels."""
        self._check(self.lib.cosenu_set_wait_limit(self.h, seconds))

    @property
    def phy_time(self) -> float:
        t = C.c_double()
        self.lib.cosenu_time(self.h, C.byref(t), None)
        return t.value

    @property
    def steps(self) -> int:
        n = C.c_longlong()
        self.lib.cosenu_time(self.h, None, C.byref(n))
        return n.value

    def analyse(self) -> dict:
        d = L.Diag()
        self._check(self.lib.cosenu_analyse(self.h, C.byref(d)))
        return d.as_dict()

    def pee_v(self) -> tuple[np.ndarray, np.ndarray]:
        a = np.zeros(self.nvz)
        b = np.zeros(self.nvz)
        self._check(self.lib.cosenu_pee_v(self.h, a.ctypes.data, b.ctypes.data))
        return a, b

    def tile(self) -> tuple[int, int]:
        tz, tv = C.c_int(), C.c_int()
        self.lib.cosenu_tile(self.h, C.byref(tz), C.byref(tv))
        return tz.value, tv.value

    def device_bytes(self) -> int:
        n = C.c_size_t()
        self.lib.cosenu_device_bytes(self.h, C.byref(n))
        return n.value

    def launches_per_step(self) -> int:
        return self.lib.cosenu_launches_per_step(self.h)

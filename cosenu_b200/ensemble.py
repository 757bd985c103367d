"""Ensembles of independent simulations advanced together on one GPU
(cosenu_batch_* of include/cosenu_b200.h), and the distribution of the
256-instance FV ensemble workload.

The reference runs one configuration per process (manage.py:361-428 submits
one job per (nz, nvz, CFL)); here hundreds of uneven instances share every
RK4 stage launch.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .nuosc import NuOsc, make_params


@dataclass
class Instance:
    """One member: grid, physics, initial-condition parameters, step count."""
    nz: int
    nvz: int
    alpha: float
    sig_nu: float
    sig_nubar: float
    mu: float
    seed: int
    nsteps: int
    z0: float = -600.0
    z1: float = 600.0
    cfl: float = 0.4
    # position in the whole workload: keys the member's random perturbation, so
    # that it does not depend on which ensemble (or rank) runs the member;
    # -1: its position in the ensemble that runs it
    index: int = -1

    @property
    def cells(self) -> int:
        return self.nz * self.nvz

    def params(self, scheme: str = "fv", precision: str = "fp64", device: int = 0) -> L.Params:
        return make_params(nz=self.nz, nvz=self.nvz, gz=4, z0=self.z0, z1=self.z1, cfl=self.cfl,
                           pmo=1.0, omega=0.0, theta_deg=0.0, mu=self.mu, scheme=scheme,
                           precision=precision, device=device)


def steps_to(t_end: float, nz: int, z0: float = -600.0, z1: float = 600.0,
             cfl: float = 0.4) -> int:
    """RK4 steps to reach t_end with dt = CFL*dz (src/nuosc.hpp:80)."""
    dt = cfl * (z1 - z0) / nz
    return int(math.ceil(t_end / dt - 1e-9))


def ensemble_instances(n: int = 256, seed: int = 20240601, t_factor: float = 1000.0,
                       nvz_choices=(32, 64, 128, 256), nz_range=(512, 8192)) -> list[Instance]:
    """The ensemble workload: nz log-uniform in [512, 8192] rounded to 256, nvz from
    {32, 64, 128, 256}, alpha ~ U[0.6, 1.2], sigma_nu ~ U[0.4, 0.8],
    sigma_nubar ~ U[0.3, 0.7], mu ~ U[0.5, 2], its own seeded +-1e-6 ex
    perturbation, run to t = t_factor / mu on z in [-600, 600]."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        nz = int(256 * round(math.exp(rng.uniform(math.log(nz_range[0]),
                                                  math.log(nz_range[1]))) / 256))
        nz = min(max(nz, 256), nz_range[1])
        nvz = int(rng.choice(nvz_choices))
        alpha = float(rng.uniform(0.6, 1.2))
        sig_nu = float(rng.uniform(0.4, 0.8))
        sig_nubar = float(rng.uniform(0.3, 0.7))
        mu = float(rng.uniform(0.5, 2.0))
        out.append(Instance(nz, nvz, alpha, sig_nu, sig_nubar, mu, seed=seed * 1000 + i,
                            nsteps=steps_to(t_factor / mu, nz), index=i))
    return out


class Ensemble:
    def __init__(self, instances: list[Instance], scheme: str = "fv", precision: str = "fp64",
                 device: int = 0):
        self.lib = L.load()
        self.instances = list(instances)
        n = len(self.instances)
        self._params = (L.Params * n)(*[x.params(scheme, precision, device) for x in instances])
        h = C.c_void_p()
        rc = self.lib.cosenu_batch_create(n, self._params, C.byref(h))
        if rc != L.OK:
            raise L.CosenuError(rc, self.lib.cosenu_last_error(None).decode())
        self.h = h
        self.members = [NuOsc._member(self.lib.cosenu_batch_member(self.h, i), self._params[i])
                        for i in range(n)]

    def _check(self, rc: int) -> None:
        if rc != L.OK:
            raise L.CosenuError(rc, self.lib.cosenu_batch_last_error(self.h).decode())

    def close(self) -> None:
        if getattr(self, "h", None):
            for m in self.members:
                m.h = None
            self.lib.cosenu_batch_destroy(self.h)
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

    def __len__(self):
        return len(self.instances)

    def init_seeded(self, amp: float = 1e-6) -> None:
        """Seeded initial conditions (cosenu_init_seeded per member); a member's
        perturbation is keyed by its seed and its index in the workload."""
        if all(x.index >= 0 for x in self.instances):
            for m, x in zip(self.members, self.instances):
                m.init_seeded(x.seed, instance=x.index, sig_nu=x.sig_nu, sig_nubar=x.sig_nubar,
                              alpha=x.alpha, amp=amp)
            return
        n = len(self)
        seeds = (C.c_uint64 * n)(*[x.seed for x in self.instances])
        d = lambda key: (C.c_double * n)(*[getattr(x, key) for x in self.instances])  # noqa: E731
        self._check(self.lib.cosenu_batch_init_seeded(self.h, seeds, d("sig_nu"), d("sig_nubar"),
                                                      d("alpha"), amp))

    def run(self, nsteps=None) -> None:
        n = len(self)
        steps = [x.nsteps for x in self.instances] if nsteps is None else list(nsteps)
        self._check(self.lib.cosenu_batch_run(self.h, (C.c_longlong * n)(*steps)))

    def set_stream(self, stream_handle: int) -> None:
        self._check(self.lib.cosenu_batch_set_stream(self.h, stream_handle))

    def synchronize(self) -> None:
        self._check(self.lib.cosenu_batch_synchronize(self.h))

    def autotune(self, trial_steps: int = 3) -> str:
        buf = C.create_string_buffer(8192)
        self._check(self.lib.cosenu_batch_autotune(self.h, trial_steps, buf, 8192))
        return buf.value.decode()

    def config(self) -> dict:
        n = len(self)
        ut, tz = C.c_int(), C.c_int()
        tv = (C.c_int * n)()
        self._check(self.lib.cosenu_batch_config(self.h, C.byref(ut), C.byref(tz), tv))
        return {"use_tma": bool(ut.value), "tz": tz.value, "tv": list(tv)}

    def set_config(self, use_tma: bool, tz: int = 32, tv=None) -> None:
        n = len(self)
        arr = (C.c_int * n)(*(tv if tv is not None else [min(64, x.nvz) for x in self.instances]))
        self._check(self.lib.cosenu_batch_set_config(self.h, int(use_tma), tz, arr))


def run_on_gpu(instances: list[Instance], precision: str = "fp64", device: int = 0,
               trial_steps: int = 3, stream=None) -> tuple[list[dict], float, dict]:
    """Runs `instances` as one batched ensemble on one GPU: seeded initial
    conditions, autotuned kernel family and tiles, every member to its own
    step count.  Returns the per-member end-of-run analysis (the keys of
    NuOsc.analyse), the device time of the run in seconds (CUDA events on the
    ensemble's stream) and the chosen kernel configuration."""
    import torch
    torch.cuda.set_device(device)
    if stream is None:
        stream = torch.cuda.Stream(device=device)
    with Ensemble(instances, precision=precision, device=device) as ens:
        ens.set_stream(stream.cuda_stream)
        ens.init_seeded()
        report = ens.autotune(trial_steps=trial_steps) if trial_steps > 0 else ""
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        torch.cuda.synchronize(device)
        e0.record(stream)
        ens.run()
        e1.record(stream)
        ens.synchronize()
        torch.cuda.synchronize(device)
        seconds = e0.elapsed_time(e1) / 1e3
        results = [m.analyse() for m in ens.members]
        cfg = ens.config()
        cfg["autotune"] = report.strip().splitlines()
    return results, seconds, cfg

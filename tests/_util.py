"""Shared helpers of the test suite (fixture loading, comparisons)."""
from __future__ import annotations

import json
import os

import numpy as np

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")


def load_golden(name: str):
    from oracle.oracle import Case
    d = np.load(os.path.join(GOLDEN, f"{name}.npz"))
    case = Case(**json.loads(str(d["case"])))
    return case, d


def text(arr) -> str:
    return bytes(np.asarray(arr, dtype=np.uint8)).decode()


def with_ghosts(case, interior: np.ndarray, oracle) -> np.ndarray:
    """Interior [..., nvz, nz] -> reference layout with ghosts filled for case.bc."""
    shp = interior.shape[:-1] + (case.ld,)
    a = np.zeros(shp)
    a[..., case.gz:case.gz + case.nz] = interior
    if a.ndim == 3:
        return oracle.fill_ghosts(case, a)
    return a


def maxabs_per_comp(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.abs(a - b).reshape(a.shape[0], -1).max(axis=1)


def gpu_from_case(case, **kw):
    from cosenu_b200 import NuOsc
    return NuOsc(nz=case.nz, nvz=case.nvz, gz=case.gz, z0=case.z0, z1=case.z1, v0=case.v0,
                 v1=case.v1, cfl=case.cfl, pmo=case.pmo, omega=case.omega,
                 theta_deg=case.theta_deg, mu=case.mu, scheme=case.scheme, bc=case.bc,
                 vac=case.vac, mat=case.mat, coll=case.coll, advec_off=case.advec_off,
                 fd_advec=case.fd_advec, ko_order=case.ko_order, **kw)

"""ctypes binding of libcosenu_b200.so (the C ABI in include/cosenu_b200.h).

The library is built in-tree by ``cosenu_b200/build.py``; importing this
module without it raises, there is no CPU fallback.
"""
from __future__ import annotations

import ctypes as C
import os

PKG = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG, "libcosenu_b200.so")

OK, ERR_ARG, ERR_CUDA, ERR_STATE, ERR_NONFINITE, ERR_NOMEM = range(6)
FV, FD = 0, 1
PERIODIC, OPEN = 0, 1
VAC, MAT, COLL, ADVEC_OFF = 1, 2, 4, 8
FD_CENTER, FD_UPWIND, FD_LOPSIDED = 0, 1, 2
FP64, FP32_BULK = 0, 1

# every symbol include/cosenu_b200.h declares
EXPORTS = (
    "cosenu_params_default", "cosenu_create", "cosenu_destroy", "cosenu_last_error",
    "cosenu_set_vac_pars", "cosenu_set_collective_pars", "cosenu_set_stream", "cosenu_grid",
    "cosenu_upload", "cosenu_download", "cosenu_set_profile", "cosenu_set_state0",
    "cosenu_mark_state0", "cosenu_step", "cosenu_step_stage", "cosenu_prepare_graphs",
    "cosenu_synchronize",
    "cosenu_time", "cosenu_analyse", "cosenu_pee_v", "cosenu_init_seeded",
    "cosenu_init_reference", "cosenu_device_state", "cosenu_upload_device",
    "cosenu_download_device", "cosenu_launches_per_step", "cosenu_tile", "cosenu_device_bytes",
    "cosenu_step_noalloc", "cosenu_snapshot", "cosenu_snapshot_wait",
    "cosenu_set_wait_limit", "cosenu_test_stall_pipeline",
    "cosenu_batch_create", "cosenu_batch_destroy", "cosenu_batch_last_error",
    "cosenu_batch_size", "cosenu_batch_member", "cosenu_batch_init_seeded", "cosenu_batch_run",
    "cosenu_batch_synchronize", "cosenu_batch_autotune", "cosenu_batch_config",
    "cosenu_batch_set_config", "cosenu_batch_set_stream",
    "cosenu_mlp_create", "cosenu_mlp_destroy", "cosenu_mlp_last_error", "cosenu_mlp_num_params",
    "cosenu_mlp_get_params", "cosenu_mlp_set_params", "cosenu_mlp_forward",
    "cosenu_mlp_loss_grad", "cosenu_mlp_set_data", "cosenu_mlp_train",
    "cosenu_mlp_set_timing", "cosenu_mlp_timing",
)


class Params(C.Structure):
    _fields_ = [("nz", C.c_int), ("nvz", C.c_int), ("gz", C.c_int),
                ("z0", C.c_double), ("z1", C.c_double), ("v0", C.c_double), ("v1", C.c_double),
                ("cfl", C.c_double), ("pmo", C.c_double), ("omega", C.c_double),
                ("theta_deg", C.c_double), ("mu", C.c_double),
                ("scheme", C.c_int), ("bc", C.c_int), ("flags", C.c_uint),
                ("fd_advec", C.c_int), ("ko_order", C.c_int), ("precision", C.c_int),
                ("device", C.c_int), ("tile_z", C.c_int), ("tile_v", C.c_int)]


class Diag(C.Structure):
    _fields_ = [(n, C.c_double) for n in ("dP_max", "avdP", "avbdP", "M0", "M0_e1", "M0_e2",
                                          "M0_e3", "Pee", "Pbee", "trace", "btrace", "eln")]

    def as_dict(self) -> dict:
        return {n: getattr(self, n) for n, _ in self._fields_}


DPTR8 = C.c_void_p * 8

_lib = None


class CosenuError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"cosenu error {code}: {msg}")
        self.code = code


def load(path: str | None = None) -> C.CDLL:
    """Loads the library (once); raises if it has not been built."""
    global _lib
    if _lib is not None:
        return _lib
    path = path or LIB_PATH
    if not os.path.exists(path):
        raise ImportError(f"{path} is missing: build it with `python cosenu_b200/build.py` "
                          "(the CUDA path has no fallback)")
    lib = C.CDLL(path)
    vp, i, d = C.c_void_p, C.c_int, C.c_double
    sig = {
        "cosenu_params_default": (None, [C.POINTER(Params)]),
        "cosenu_create": (i, [C.POINTER(Params), C.POINTER(vp)]),
        "cosenu_destroy": (i, [vp]),
        "cosenu_last_error": (C.c_char_p, [vp]),
        "cosenu_set_vac_pars": (i, [vp, d, d, d]),
        "cosenu_set_collective_pars": (i, [vp, d]),
        "cosenu_set_stream": (i, [vp, vp]),
        "cosenu_grid": (i, [vp, C.POINTER(d)]),
        "cosenu_upload": (i, [vp, DPTR8, i]),
        "cosenu_download": (i, [vp, DPTR8, i]),
        "cosenu_set_profile": (i, [vp, vp, vp, i]),
        "cosenu_set_state0": (i, [vp, DPTR8, i]),
        "cosenu_mark_state0": (i, [vp]),
        "cosenu_step": (i, [vp, i]),
        "cosenu_step_stage": (i, [vp, i]),
        "cosenu_prepare_graphs": (i, [vp]),
        "cosenu_synchronize": (i, [vp]),
        "cosenu_set_wait_limit": (i, [vp, d]),
        "cosenu_test_stall_pipeline": (i, [vp, i]),
        "cosenu_time": (i, [vp, C.POINTER(d), C.POINTER(C.c_longlong)]),
        "cosenu_analyse": (i, [vp, C.POINTER(Diag)]),
        "cosenu_pee_v": (i, [vp, vp, vp]),
        "cosenu_init_seeded": (i, [vp, C.c_uint64, C.c_uint32, d, d, d, d]),
        "cosenu_init_reference": (i, [vp, d]),
        "cosenu_device_state": (i, [vp, C.c_void_p * 8, C.POINTER(i)]),
        "cosenu_upload_device": (i, [vp, DPTR8, i]),
        "cosenu_download_device": (i, [vp, DPTR8, i]),
        "cosenu_launches_per_step": (i, [vp]),
        "cosenu_tile": (i, [vp, C.POINTER(i), C.POINTER(i)]),
        "cosenu_device_bytes": (i, [vp, C.POINTER(C.c_size_t)]),
        "cosenu_step_noalloc": (i, [C.POINTER(Params), DPTR8, i, i, vp]),
        "cosenu_snapshot": (i, [vp, C.POINTER(C.c_longlong)]),
        "cosenu_snapshot_wait": (i, [vp, C.POINTER(C.POINTER(d))]),
        "cosenu_batch_create": (i, [i, C.POINTER(Params), C.POINTER(vp)]),
        "cosenu_batch_destroy": (i, [vp]),
        "cosenu_batch_last_error": (C.c_char_p, [vp]),
        "cosenu_batch_size": (i, [vp]),
        "cosenu_batch_member": (vp, [vp, i]),
        "cosenu_batch_init_seeded": (i, [vp, vp, vp, vp, vp, d]),
        "cosenu_batch_run": (i, [vp, vp]),
        "cosenu_batch_synchronize": (i, [vp]),
        "cosenu_batch_autotune": (i, [vp, i, C.c_char_p, C.c_size_t]),
        "cosenu_batch_config": (i, [vp, C.POINTER(i), C.POINTER(i), vp]),
        "cosenu_batch_set_config": (i, [vp, i, i, vp]),
        "cosenu_batch_set_stream": (i, [vp, vp]),
        "cosenu_mlp_create": (i, [i, i, i, i, C.c_uint64, i, C.POINTER(vp)]),
        "cosenu_mlp_destroy": (i, [vp]),
        "cosenu_mlp_last_error": (C.c_char_p, [vp]),
        "cosenu_mlp_num_params": (i, [vp, C.POINTER(C.c_size_t)]),
        "cosenu_mlp_get_params": (i, [vp, vp]),
        "cosenu_mlp_set_params": (i, [vp, vp]),
        "cosenu_mlp_forward": (i, [vp, vp, i, vp]),
        "cosenu_mlp_loss_grad": (i, [vp, vp, vp, i, C.POINTER(C.c_float), vp]),
        "cosenu_mlp_set_data": (i, [vp, vp, vp, i]),
        "cosenu_mlp_train": (i, [vp, i, i, C.c_float, C.c_float, C.c_float, C.c_float,
                                 C.c_float, C.c_uint64, vp]),
        "cosenu_mlp_set_timing": (i, [vp, i]),
        "cosenu_mlp_timing": (i, [vp, C.POINTER(d)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    _lib = lib
    return lib


def default_params() -> Params:
    p = Params()
    load().cosenu_params_default(C.byref(p))
    return p

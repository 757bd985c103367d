"""cosenu_step_noalloc: the entry point for callers that must not allocate
device memory (their device memory all comes from their own pool, or their
loop cannot take the device synchronisation a cudaMalloc/cudaFree may cause).

The caller holds the state in its own device memory (here: torch tensors, the
test's memory, not the library's); the entry point advances it using only the
library's fixed scratch array.  Its result must equal what the context-based
path (cosenu_create / cosenu_upload / cosenu_step) computes, within the
1e-12 max-abs tolerance the other parity tests use, on two calls in a row
(the second call starts from the first call's output and reuses the scratch).

This file is collected last so that a failure here comes after every other
test has run; it passes alone in a fresh process as well.
"""
import ctypes as C

import numpy as np
import pytest

from cosenu_b200 import NuOsc, make_params
from cosenu_b200 import _lib as L

TOL = 1e-12


def _call(p, dev, ld, nsteps):
    lib = L.load()
    ptrs = L.DPTR8(*[dev[c].data_ptr() for c in range(8)])
    rc = lib.cosenu_step_noalloc(C.byref(p), ptrs, ld, nsteps, None)
    assert rc == L.OK, lib.cosenu_last_error(None).decode()


FD_SMALL = dict(scheme="fd", nz=512, nvz=48, gz=2, omega=1e-3, theta_deg=1e-6, z0=-256.0,
                z1=256.0)
T32x16 = dict(tile_z=32, tile_v=16)


@pytest.mark.gpu
@pytest.mark.parametrize("kw,tiles,pad", [
    (dict(scheme="fv", nz=1024, nvz=64, gz=4, omega=0.0), T32x16, 0),  # the small FV grid
    (FD_SMALL, T32x16, 0),
    (dict(scheme="fv", nz=256, nvz=20, gz=4, bc="open", omega=1e-2, theta_deg=37.0, z0=-128.0,
          z1=128.0), T32x16, 0),
    # the default v tile (min(nvz, 64)) and a collective-term-free run
    (dict(FD_SMALL, nvz=96), {}, 0),
    (dict(FD_SMALL, coll=False), T32x16, 0),
    # FP32-bulk: the increments and the second state buffer in the scratch
    (dict(FD_SMALL, precision="fp32"), T32x16, 0),
    (dict(scheme="fv", nz=256, nvz=20, gz=4, omega=1e-2, theta_deg=37.0, z0=-128.0, z1=128.0,
          precision="fp32"), T32x16, 0),
    # the upwind FD stencil (its row factors come from the scratch tables)
    (dict(FD_SMALL, fd_advec="upwind", ko_order=5, gz=3), dict(tile_z=16, tile_v=5), 0),
    # rows of the caller's tensor padded past nz (row pitch ld = nz + 8)
    (dict(scheme="fv", nz=256, nvz=20, gz=4, omega=1e-2, theta_deg=37.0, z0=-128.0, z1=128.0),
     T32x16, 8),
])
def test_step_noalloc_matches_context_path(kw, tiles, pad):
    import torch
    nz, gz = kw["nz"], kw["gz"]
    ld = nz + pad
    ref = NuOsc(**kw, **tiles)
    ref.init_seeded(7)
    st0 = ref.download()
    # caller-owned device state: [8][nvz][ld], interior at [..., :nz]
    host = np.zeros((8, kw["nvz"], ld))
    host[:, :, :nz] = st0[:, :, gz:gz + nz]
    dev = torch.tensor(host, device="cuda")
    p = make_params(**kw, **tiles)
    for call in range(2):
        _call(p, dev, ld, 9)
        torch.cuda.synchronize()
        ref.evolve(9)
        want = ref.download()[:, :, gz:gz + nz]
        got = dev.cpu().numpy()
        err = np.abs(got[:, :, :nz] - want).max()
        assert err <= TOL, (call, err)
        assert np.isfinite(got).all()
        assert not got[:, :, nz:].any()  # the row padding is left alone
    ref.close()


def test_step_noalloc_rejects_grids_beyond_its_scratch():
    """Checked before any device work, so this runs without a GPU too."""
    lib = L.load()
    p = make_params(nz=4096, nvz=64)  # 64 * 4128 padded cells > 69632
    ptrs = L.DPTR8(*([1] * 8))  # never dereferenced: the size check comes first
    rc = lib.cosenu_step_noalloc(C.byref(p), ptrs, 4096, 1, None)
    assert rc == L.ERR_ARG
    msg = lib.cosenu_last_error(None).decode()
    assert "69632" in msg and "too large" in msg

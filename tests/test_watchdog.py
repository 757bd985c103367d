"""The stage kernels' pipeline watchdog.

Every wait inside the TMA-pipelined stage kernel is bounded in time; when one
runs out the kernel records an error word, carries on along the same control
path and the host reports COSENU_ERR_CUDA.  These tests make the waits run
out without a fault or a hang: with the stall hook the producer warp issues no
copies, so the consumers' full barriers are never completed, their waits (a
1 ms limit here) expire, and nothing is in flight when the blocks exit.  The
context then works again after a new state is uploaded.
"""
import ctypes as C

import numpy as np
import pytest

from tests._util import gpu_from_case

pytestmark = pytest.mark.gpu


def _case(scheme):
    from oracle.oracle import Case
    return Case(nz=4096, nvz=37, gz=4 if scheme == "fv" else 2, z0=-2048.0, z1=2048.0,
                scheme=scheme, omega=1e-2, theta_deg=37.0, mu=1.0)


@pytest.mark.parametrize("nsteps", [1, 17])  # direct launches and a captured graph
@pytest.mark.parametrize("scheme", ["fd", "fv"])
def test_expired_wait_is_reported_and_context_recovers(gpu_lib, oracle, monkeypatch, scheme,
                                                       nsteps):
    from cosenu_b200._lib import ERR_CUDA, CosenuError
    monkeypatch.setenv("COSENU_KERNEL", "tma")
    case = _case(scheme)
    G, bG, st0 = oracle.init_seeded(case, seed=3)
    with gpu_from_case(case) as sim:
        sim.upload(st0)
        sim.set_wait_limit(1e-3)
        assert gpu_lib.cosenu_test_stall_pipeline(sim.h, 1) == 0
        sim.evolve(nsteps)
        with pytest.raises(CosenuError) as e:
            sim.synchronize()
        assert e.value.code == ERR_CUDA and "timed out" in str(e.value)
        # the report repeats until a new state arrives
        with pytest.raises(CosenuError) as e:
            sim.download()
        assert e.value.code == ERR_CUDA
        # normal operation again: no stall, a new state, results as the oracle's
        assert gpu_lib.cosenu_test_stall_pipeline(sim.h, 0) == 0
        sim.set_wait_limit(2.0)
        sim.upload(st0)
        sim.evolve(5)
        sim.synchronize()
        got = sim.download()
    ref = oracle.step(case, st0, 5)
    assert np.abs(got - ref).max() <= 1e-12


def test_stall_hook_needs_the_tma_kernel(gpu_lib, oracle, monkeypatch):
    from cosenu_b200._lib import ERR_STATE
    monkeypatch.setenv("COSENU_KERNEL", "ldg")
    case = _case("fd")
    with gpu_from_case(case) as sim:
        assert gpu_lib.cosenu_test_stall_pipeline(sim.h, 1) == ERR_STATE


def test_wait_limit_range(gpu_lib):
    from cosenu_b200._lib import ERR_ARG
    case = _case("fd")
    with gpu_from_case(case) as sim:
        assert gpu_lib.cosenu_set_wait_limit(sim.h, 0.0) == ERR_ARG
        assert gpu_lib.cosenu_set_wait_limit(sim.h, 1e4) == ERR_ARG
        assert gpu_lib.cosenu_set_wait_limit(sim.h, 0.5) == 0

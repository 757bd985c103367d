"""The GPU path's RK4 update order, restated in numpy on the oracle's
right-hand side (CPU): with FP64 stage values it forms the accumulator once,
in stage 3, from differences of stored stage values,
    U = Y + dt/2 k1,  U' = Y + dt/2 k2,  U'' = Y + dt k3,
    A = Y + (U - Y)/3 + 2 (U' - Y)/3 + dt/3 k3,  Y <- A + dt/6 k4,
instead of updating it at every stage (src/nuosc.hpp:281-318, restated by
the oracle's step).  The two orders must agree to rounding."""
import numpy as np
import pytest

from tests._util import load_golden, with_ghosts


def _deferred_steps(oracle, case, y, n):
    dt = case.dt
    g = slice(case.gz, case.gz + case.nz)
    for _ in range(n):
        u = y + 0.5 * dt * oracle.rhs(case, y)
        u1 = y + 0.5 * dt * oracle.rhs(case, u)
        k3 = oracle.rhs(case, u1)
        u2 = y + dt * k3
        a = y + (u - y) * (1.0 / 3.0) + (u1 - y) * (2.0 / 3.0) + (dt / 3.0) * k3
        y = a + (dt / 6.0) * oracle.rhs(case, u2)
        y = oracle.fill_ghosts(case, np.where(np.arange(case.ld) < case.gz, 0.0, y))
    return y[..., g]


@pytest.mark.parametrize("name", ["fv_small", "fd_small", "fv_open", "fd_mat"])
def test_deferred_accumulator_equals_reference_order(oracle, name):
    case, d = load_golden(name)
    st0 = with_ghosts(case, d["state0"], oracle)
    n = int(d["dump_steps"][-1])
    ref = oracle.step(case, st0, n)[..., case.gz:case.gz + case.nz]
    got = _deferred_steps(oracle, case, st0, n)
    assert np.abs(got - ref).max() <= 1e-13
    # and both reproduce what the reference binary wrote
    assert np.abs(got - d[f"rho_{n}"]).max() <= 1e-10

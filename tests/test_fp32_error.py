"""Error of the FP32-bulk form (FP32 stage increments over an FP64 base state)
against the FP64 oracle and the reference's own runs.

Bounds, with the values measured on a B200 in brackets:
* the 1024 x 64 FV grid, 500 steps (before saturation), against the oracle's
  FP64 state: max-abs per component <= 5e-9 [7.6e-10 for ex, 1.3e-11 for
  ee / xx]; <P_ee>(t), <P_ee-bar>(t) every 50 steps <= 1e-11 [9e-13]; trace and
  ELN drift <= 1e-12 relative [2e-14];
* the same grid through saturation (1500 steps), against the reference's
  analysis rows: <P_ee>, <P_ee-bar>, |M0| and P_ee(v) <= 1e-6 [<= 1e-7; the
  rows carry 7 digits], trace and ELN drift <= 1e-8 [5e-10];
* the FD benchmark grid (nz 32768 x nvz 256), 10 steps, against the
  reference's dumps: <= 1e-12 per component [3e-14].
"""
import numpy as np
import pytest

from tests._util import gpu_from_case, load_golden, maxabs_per_comp

pytestmark = pytest.mark.gpu


def _i(case, a):
    return a[..., case.gz:case.gz + case.nz]


def test_fp32_bulk_before_saturation_against_fp64_oracle(gpu_lib, oracle):
    case, d = load_golden("c1_pre")
    G, bG, st0 = oracle.init_seeded(case, seed=int(d["seed"]))
    ref, ref_an = st0, []
    for _ in range(10):
        ref = oracle.step(case, ref, 50)
        ref_an.append(oracle.analyse(case, ref, G, bG, st0))
    with gpu_from_case(case, precision="fp32") as sim:
        sim.init_seeded(int(d["seed"]))
        a0 = sim.analyse()
        an = []
        for _ in range(10):
            sim.evolve(50)
            an.append(sim.analyse())
        got = sim.download()
    err = maxabs_per_comp(_i(case, got), _i(case, ref))
    assert np.all(err <= 5e-9), err
    for a, b in zip(an, ref_an):
        assert abs(a["Pee"] - b["Pee"]) <= 1e-11 and abs(a["Pbee"] - b["Pbee"]) <= 1e-11
    for k in ("trace", "btrace", "eln"):
        assert abs(an[-1][k] - a0[k]) <= 1e-12 * abs(a0[k]), k


def test_fp32_bulk_after_saturation_against_reference(gpu_lib):
    case, d = load_golden("c1_sat")
    with gpu_from_case(case, precision="fp32") as sim:
        sim.init_seeded(int(d["seed"]))
        a0 = sim.analyse()
        t_prev = 0
        worst = 0.0
        for row, row_sp in zip(d["conserved_quantities"], d["survival_probability"]):
            t = int(row[0])
            sim.evolve(t - t_prev)
            t_prev = t
            a = sim.analyse()
            worst = max(worst, abs(a["Pee"] - row_sp[1]), abs(a["Pbee"] - row_sp[2]),
                        abs(a["M0"] - row[4]))
        pee, pbee = sim.pee_v()
    assert d["survival_probability"][-1][1] < 0.9  # the run did saturate
    assert worst <= 1e-6, worst
    assert np.abs(pee - d["rho_1500_pee_v"]).max() <= 1e-6
    assert np.abs(pbee - d["rho_1500_pbee_v"]).max() <= 1e-6
    for k in ("trace", "btrace", "eln"):
        assert abs(a[k] - a0[k]) <= 1e-8 * abs(a0[k]), k


def test_fp32_bulk_benchmark_grid_against_reference(gpu_lib):
    case, d = load_golden("c2_ref")
    cols = d["columns"]
    with gpu_from_case(case, precision="fp32") as sim:
        sim.init_seeded(int(d["seed"]))
        t_prev = 0
        for t in [int(x) for x in d["dump_steps"]]:
            sim.evolve(t - t_prev)
            t_prev = t
            got = _i(case, sim.download())
            err = maxabs_per_comp(got[:, :, cols], d[f"rho_{t}_columns"])
            assert np.all(err <= 1e-12), (t, err)


def test_fp32_bulk_large_fv_grid_against_reference(gpu_lib):
    """The FV grid of the FP32-bulk workload (nz 65536 x nvz 512), 5 steps,
    against the reference's own dump: <= 1e-11 per component."""
    case, d = load_golden("c3_ref")
    cols = d["columns"]
    with gpu_from_case(case, precision="fp32") as sim:
        sim.init_seeded(int(d["seed"]))
        sim.evolve(5)
        got = _i(case, sim.download())
    err = maxabs_per_comp(got[:, :, cols], d["rho_5_columns"])
    assert np.all(err <= 1e-11), err

"""Parity of the CUDA path (through the C ABI) with the reference.

Tolerances (max-abs per component, FP64): <= 1e-10 before saturation
against the reference's own outputs (tests/golden) and against the CPU oracle;
<= 1e-6 on survival probabilities and the conservation diagnostics after
saturation.  Measured differences are far smaller (1e-14 and below).
"""
import os

import numpy as np
import pytest

from tests._util import gpu_from_case, load_golden, maxabs_per_comp, with_ghosts

pytestmark = pytest.mark.gpu

SMALL = ["fv_small", "fv_vac", "fv_oddv", "fd_small", "fd_vac", "fv_open", "fd_open", "fv_mat",
         "fd_mat", "fd_ko5", "fv_advoff", "fd_advoff"]
TOL_PRE = 1e-10
TOL_POST = 1e-6
NTHREADS = os.cpu_count() or 1


def _inputs(case, d, oracle):
    st0 = with_ghosts(case, d["state0"], oracle)
    G = with_ghosts(case, d["G"][None], oracle)[0]
    bG = with_ghosts(case, d["bG"][None], oracle)[0]
    return st0, G, bG


def _interior(case, a):
    return a[..., case.gz:case.gz + case.nz]


@pytest.mark.parametrize("kernel", ["auto", "tma"])
@pytest.mark.parametrize("name", SMALL)
def test_snapshots_match_reference(gpu_lib, oracle, name, kernel, monkeypatch):
    """Every rho_<t>.dat the reference wrote, to <= 1e-10 max-abs, with the
    default kernel choice and with the TMA-pipelined kernel forced."""
    case, d = load_golden(name)
    if kernel == "tma":
        if case.nz % 32:
            pytest.skip("the TMA kernel needs nz % 32 == 0")
        monkeypatch.setenv("COSENU_KERNEL", "tma")
    st0, G, bG = _inputs(case, d, oracle)
    with gpu_from_case(case) as sim:
        sim.upload(st0)
        t_prev = 0
        for t in d["dump_steps"]:
            sim.evolve(int(t) - t_prev)
            t_prev = int(t)
            got = _interior(case, sim.download())
            err = maxabs_per_comp(got, d[f"rho_{t}"])
            assert np.all(err <= TOL_PRE), (name, int(t), err)


@pytest.mark.parametrize("env", [{"COSENU_TMA_MINB": "1"}, {"COSENU_TMA_RING": "2"},
                                 {"COSENU_TMA_RING": "4"}])
def test_tuning_switches_keep_results(gpu_lib, env):
    """The kernel-shape switches (FV blocks per SM, FD ring depth) change
    only the schedule: results still match the reference's snapshots."""
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    p = subprocess.run([sys.executable, "-m", "tests._env_case", "fv_small", "fd_small",
                        "fv_open", "fd_open", "fv_mat"], cwd=root, capture_output=True,
                       text=True, timeout=600, env={**os.environ, **env})
    assert p.returncode == 0, p.stdout + p.stderr


@pytest.mark.parametrize("name", ["fv_small", "fd_small", "fv_vac", "fd_vac", "fv_open",
                                  "fd_ko5", "fv_mat"])
def test_analysis_matches_reference_tables(gpu_lib, oracle, name):
    """conserved_quantities.dat / survival_probability.dat rows."""
    case, d = load_golden(name)
    st0, G, bG = _inputs(case, d, oracle)
    with gpu_from_case(case) as sim:
        sim.upload(st0)
        sim.set_profile(G, bG)
        sim.set_state0(st0)
        t_prev = 0
        for row, row_sp in zip(d["conserved_quantities"], d["survival_probability"]):
            t = int(row[0])
            sim.evolve(t - t_prev)
            t_prev = t
            a = sim.analyse()
            got = np.array([a["dP_max"], a["avdP"], a["avbdP"], a["M0"]])
            # dP statistics are differences of |P| ~ 1 values: absolute tolerance
            assert np.all(np.abs(got - row[1:]) <= 1e-12 * np.maximum(np.abs(row[1:]), 1.0)), \
                (t, got, row)
            assert abs(a["Pee"] - row_sp[1]) <= 5e-7 * row_sp[1]
            assert abs(a["Pbee"] - row_sp[2]) <= 5e-7 * row_sp[2]


@pytest.mark.parametrize("tile", [(8, 1), (8, 3), (8, 32), (16, 5), (16, 16), (32, 7), (32, 16)])
@pytest.mark.parametrize("name", ["fv_vac", "fd_vac", "fv_open", "fd_open"])
def test_tile_shapes_against_oracle(gpu_lib, oracle, name, tile):
    """Any tile shape, including v tiles that do not divide nvz."""
    case, d = load_golden(name)
    st0, G, bG = _inputs(case, d, oracle)
    ref = oracle.step(case, st0, 10)
    with gpu_from_case(case, tile_z=tile[0], tile_v=tile[1]) as sim:
        assert sim.tile() == tile
        sim.upload(st0)
        sim.evolve(10)
        got = sim.download()
    err = maxabs_per_comp(_interior(case, got), _interior(case, ref))
    assert np.all(err <= 1e-12), err
    # ghost cells as updateBufferZone leaves them
    assert np.abs(got - ref).max() <= 1e-12


def test_deterministic_and_graph_equals_stagewise(gpu_lib, oracle):
    case, d = load_golden("fv_vac")
    st0, _, _ = _inputs(case, d, oracle)
    outs = []
    for mode in ("graph", "graph", "stages"):
        with gpu_from_case(case) as sim:
            sim.upload(st0)
            if mode == "graph":
                sim.evolve(37)
            else:
                for _ in range(37):
                    for s in range(4):
                        sim.step_stage(s)
            outs.append(sim.download())
    assert np.array_equal(outs[0], outs[1])
    assert np.array_equal(outs[0], outs[2])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("kernel", ["auto", "tma"])
def test_prepared_graphs_equal_lazy_capture(gpu_lib, oracle, monkeypatch, precision, kernel):
    """cosenu_prepare_graphs captures the graphs of both state-buffer parities
    ahead of use (idempotent, also with the parity flipped by an odd step
    count); stepping through them equals the lazily captured ones."""
    if kernel == "tma":
        monkeypatch.setenv("COSENU_KERNEL", "tma")
    case, d = load_golden("fv_vac")
    st0, _, _ = _inputs(case, d, oracle)
    outs = []
    for prep in (False, True):
        with gpu_from_case(case, precision=precision) as sim:
            sim.upload(st0)
            if prep:
                sim.prepare_graphs()
                sim.prepare_graphs()
            sim.evolve(3)
            if prep:
                sim.prepare_graphs()
            sim.evolve(37)
            outs.append(sim.download())
    assert np.array_equal(outs[0], outs[1])


def test_snapshot_is_the_state_at_the_call(gpu_lib, oracle):
    """cosenu_snapshot: the host copy holds the state at the call even when
    more steps are queued before cosenu_snapshot_wait; consecutive snapshots
    reuse the buffers."""
    case, d = load_golden("fv_vac")
    st0, _, _ = _inputs(case, d, oracle)
    with gpu_from_case(case) as sim:
        sim.upload(st0)
        sim.evolve(5)
        assert sim.snapshot() == 5
        sim.evolve(11)
        snap5 = sim.snapshot_wait()
        ref16 = _interior(case, sim.download())
        assert sim.snapshot() == 16
        snap16 = sim.snapshot_wait()
    ref5 = oracle.step(case, st0, 5)
    assert np.array_equal(snap16, ref16)
    assert maxabs_per_comp(snap5, _interior(case, ref5)).max() <= 1e-10
    assert not np.array_equal(snap5, snap16)


def test_device_initial_conditions_bitwise(gpu_lib, oracle):
    """On-device seeded and reference initial conditions equal the host
    recipes bit for bit."""
    case, d = load_golden("c1_pre")
    G, bG, st = oracle.init_seeded(case, seed=int(d["seed"]))
    with gpu_from_case(case) as sim:
        sim.init_seeded(int(d["seed"]))
        got = sim.download()
    assert np.array_equal(_interior(case, got), _interior(case, st))
    case, d = load_golden("fv_default_ic")
    with gpu_from_case(case) as sim:
        sim.initialize(float(d["perturbation_size"]))
        got = sim.download()
    assert np.array_equal(np.moveaxis(_interior(case, got), 0, -1), d["state0"])


def _c1(oracle, name):
    case, d = load_golden(name)
    G, bG, st0 = oracle.init_seeded(case, seed=int(d["seed"]))
    return case, d, G, bG, st0


def test_c1_pre_saturation_500_steps(gpu_lib, oracle):
    """The small FV workload as specified (WENO7, 1024 x 64, 500 steps): against the
    reference run (subset, checksums, analysis rows) and the full oracle
    state, <= 1e-10 max-abs per component."""
    case, d, G, bG, st0 = _c1(oracle, "c1_pre")
    with gpu_from_case(case) as sim:
        sim.init_seeded(int(d["seed"]))
        t_prev = 0
        for row, row_sp in zip(d["conserved_quantities"], d["survival_probability"]):
            t = int(row[0])
            sim.evolve(t - t_prev)
            t_prev = t
            a = sim.analyse()
            assert abs(a["M0"] - row[4]) <= 1e-10
            assert abs(a["dP_max"] - row[1]) <= 1e-10
            assert abs(a["Pee"] - row_sp[1]) <= 5e-7 and abs(a["Pbee"] - row_sp[2]) <= 5e-7
        got = _interior(case, sim.download())
        pee, pbee = sim.pee_v()
    err = maxabs_per_comp(got[:, :, ::16], d["rho_500_subset"])
    assert np.all(err <= TOL_PRE), err
    ck = np.stack([got.sum(axis=(1, 2)), (got * got).sum(axis=(1, 2)),
                   np.abs(got).sum(axis=(1, 2))], 1)
    assert np.allclose(ck, d["rho_500_checksums"], rtol=1e-10, atol=1e-14)
    assert np.abs(pee - d["rho_500_pee_v"]).max() <= 1e-10
    ref = oracle.step(case, st0, 500, nthreads=NTHREADS)
    err = maxabs_per_comp(got, _interior(case, ref))
    assert np.all(err <= TOL_PRE), err


def test_c1_after_saturation_1500_steps(gpu_lib, oracle):
    """The 1024 x 64 FV grid through saturation: <Pee>, <Pbee>, |M0|, max dP and
    P_ee(v) against the reference run at every analysis step, <= 1e-6."""
    case, d, G, bG, st0 = _c1(oracle, "c1_sat")
    worst = 0.0
    with gpu_from_case(case) as sim:
        sim.init_seeded(int(d["seed"]))
        t_prev = 0
        for row, row_sp in zip(d["conserved_quantities"], d["survival_probability"]):
            t = int(row[0])
            sim.evolve(t - t_prev)
            t_prev = t
            a = sim.analyse()
            for got, want in ((a["Pee"], row_sp[1]), (a["Pbee"], row_sp[2]), (a["M0"], row[4]),
                              (a["dP_max"], row[1]), (a["avdP"], row[2]), (a["avbdP"], row[3])):
                worst = max(worst, abs(got - want))
        pee, pbee = sim.pee_v()
    assert d["survival_probability"][-1][1] < 0.9  # the run did saturate
    assert worst <= TOL_POST, worst
    assert np.abs(pee - d["rho_1500_pee_v"]).max() <= TOL_POST
    assert np.abs(pbee - d["rho_1500_pbee_v"]).max() <= TOL_POST


def test_c2_full_size_one_step_and_conservation(gpu_lib, oracle):
    """The large FD grid (32768 x 256): one step at full size against the
    oracle, then trace, anti-trace and ELN conservation over further steps
    (omega sin 2 theta ~ 3e-11 leaves ELN conserved far below the bound)."""
    from oracle.oracle import Case
    case = Case(nz=32768, nvz=256, gz=2, z0=-3000.0, z1=3000.0, scheme="fd", pmo=1.0,
                omega=1e-3, theta_deg=1e-6, mu=1.0)
    G, bG, st0 = oracle.init_seeded(case, seed=7)
    ref = oracle.step(case, st0, 1, nthreads=NTHREADS)
    with gpu_from_case(case) as sim:
        sim.init_seeded(7)
        sim.evolve(1)
        got = sim.download()
        err = maxabs_per_comp(_interior(case, got), _interior(case, ref))
        assert np.all(err <= 1e-12), err
        a0 = sim.analyse()
        sim.evolve(50)
        a1 = sim.analyse()
    assert abs(a1["trace"] - a0["trace"]) <= 1e-12 * abs(a0["trace"])
    assert abs(a1["btrace"] - a0["btrace"]) <= 1e-12 * abs(a0["btrace"])
    assert abs(a1["eln"] - a0["eln"]) <= 1e-12 * abs(a0["eln"])


def test_errors_are_reported_not_fatal(gpu_lib, oracle):
    from cosenu_b200 import NuOsc
    from cosenu_b200._lib import CosenuError, ERR_ARG, ERR_STATE, ERR_NONFINITE
    with pytest.raises(CosenuError) as e:
        NuOsc(nz=60, nvz=8)
    assert e.value.code == ERR_ARG
    case, d = load_golden("fv_small")
    st0, G, bG = _inputs(case, d, oracle)
    with gpu_from_case(case) as sim:
        with pytest.raises(CosenuError) as e:
            sim.evolve(1)
        assert e.value.code == ERR_STATE
        bad = st0.copy()
        bad[0, 3, case.gz + 5] = np.nan
        sim.upload(bad)
        sim.set_profile(G, bG)
        sim.set_state0(st0)
        sim.evolve(2)
        with pytest.raises(CosenuError) as e:
            sim.analyse()
        assert e.value.code == ERR_NONFINITE
        # the context stays usable
        sim.upload(st0)
        sim.evolve(2)
        assert np.isfinite(sim.analyse()["M0"])


@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("bc", ["periodic", "open"])
@pytest.mark.parametrize("scheme", ["fd", "fv"])
def test_tma_path_equals_register_path(gpu_lib, oracle, scheme, precision, bc):
    """The TMA-pipelined kernel (default when nz is a multiple of 32) and the
    register-tiled kernel with the same 32 x nvz tile do the same arithmetic
    in the same order: bitwise equal in FP64.  nvz = 37 leaves a partial
    8-row chunk and puts rows of both signs of v in one chunk."""
    from oracle.oracle import Case
    case = Case(nz=8192, nvz=37, gz=4 if scheme == "fv" else 2, z0=-4096.0, z1=4096.0,
                scheme=scheme, bc=bc, omega=1e-2, theta_deg=37.0, mu=1.0)
    outs = []
    for tiles in ({}, {"tile_z": 32, "tile_v": 37}):
        with gpu_from_case(case, precision=precision, **tiles) as sim:
            sim.init_seeded(11)
            sim.evolve(25)
            outs.append(sim.download())
            outs.append(sim.analyse()["M0"])
    if precision == "fp64":
        # same operations up to FMA contraction and the order of the
        # velocity-moment partial sums
        assert np.abs(outs[0] - outs[2]).max() <= 1e-13
        assert abs(outs[1] - outs[3]) <= 1e-12
    else:
        # two different kernels: FP32 rounding (contraction) may differ
        assert np.abs(outs[0] - outs[2]).max() <= 1e-6 * np.abs(outs[2]).max()
    if precision == "fp64":
        G, bG, st0 = oracle.init_seeded(case, seed=11)
        ref = oracle.step(case, st0, 25, nthreads=NTHREADS)
        assert np.abs(outs[0] - ref).max() <= 1e-12


@pytest.mark.parametrize("fd_advec", ["upwind", "lopsided"])
@pytest.mark.parametrize("tiles", [{}, {"tile_z": 16, "tile_v": 5}])
def test_fd_variants_without_reference_build_against_oracle(gpu_lib, oracle, fd_advec, tiles):
    """ADVEC_UPWIND and the lopsided stencil (src/rhs_fd.hpp:63-72) do not
    compile in the reference (undefined sgn); checked against the oracle."""
    from oracle.oracle import Case
    case = Case(nz=256, nvz=24, gz=3, z0=-128.0, z1=128.0, scheme="fd", fd_advec=fd_advec,
                ko_order=5, omega=1e-2, theta_deg=37.0)
    G, bG, st0 = oracle.init_seeded(case, seed=5)
    ref = oracle.step(case, st0, 20)
    with gpu_from_case(case, **tiles) as sim:
        sim.upload(st0)
        sim.evolve(20)
        got = sim.download()
    assert np.abs(_interior(case, got) - _interior(case, ref)).max() <= 1e-12

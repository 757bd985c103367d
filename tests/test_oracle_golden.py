"""Pins the CPU oracle (oracle/cosenu_oracle.c) to the reference.

tests/golden/*.npz hold what the reference binary (compiled from its own
sources by oracle/build.py and run by tests/golden/make_golden.py) wrote for
seeded inputs: rho_<t>.dat snapshots (16 significant digits),
survival_probability.dat and conserved_quantities.dat.  The oracle, run on
the same inputs, must reproduce them:
  * direct collective form: to the print precision (it keeps the reference's
    operand order, so it is the reference's arithmetic);
  * velocity-moment form (the form the GPU uses): <= 1e-12 max-abs.
"""
import hashlib
import os

import numpy as np
import pytest

from tests._util import load_golden, text, with_ghosts

SMALL = ["fv_small", "fv_vac", "fv_oddv", "fd_small", "fd_vac", "fv_open", "fd_open", "fv_mat",
         "fd_mat", "fd_ko5", "fv_advoff", "fd_advoff"]


def _state0(case, d, oracle):
    return with_ghosts(case, d["state0"], oracle), with_ghosts(case, d["G"][None], oracle)[0], \
        with_ghosts(case, d["bG"][None], oracle)[0]


def _print_close(a, b):
    """a equals b to the 16 significant digits of the reference's dump."""
    return np.all(np.abs(a - b) <= 2e-15 * np.abs(b) + 1e-300)


@pytest.mark.parametrize("name", SMALL)
def test_oracle_direct_matches_reference_snapshots(oracle, name):
    case, d = load_golden(name)
    st0, G, bG = _state0(case, d, oracle)
    y, t_prev = st0, 0
    for t in d["dump_steps"]:
        y = oracle.step(case, y, int(t) - t_prev, coll_direct=True)
        t_prev = int(t)
        got = y[:, :, case.gz:case.gz + case.nz]
        assert _print_close(got, d[f"rho_{t}"]), f"{name} step {t}"


@pytest.mark.parametrize("name", SMALL)
def test_oracle_moment_form_matches_reference(oracle, name):
    case, d = load_golden(name)
    st0, G, bG = _state0(case, d, oracle)
    t = int(d["dump_steps"][-1])
    y = oracle.step(case, st0, t, coll_direct=False)
    err = np.abs(y[:, :, case.gz:case.gz + case.nz] - d[f"rho_{t}"]).max()
    assert err <= 1e-12, err


@pytest.mark.parametrize("name", ["fv_small", "fd_small", "fv_vac", "fv_open", "fd_ko5"])
def test_oracle_analysis_matches_reference_tables(oracle, name):
    """conserved_quantities.dat (dcon) and survival_probability.dat rows."""
    case, d = load_golden(name)
    st0, G, bG = _state0(case, d, oracle)
    cq = d["conserved_quantities"]
    sp = d["survival_probability"]
    y, t_prev = st0, 0
    for row_cq, row_sp in zip(cq, sp):
        t = int(row_cq[0])
        y = oracle.step(case, y, t - t_prev, coll_direct=True)
        t_prev = t
        a = oracle.analyse(case, y, G, bG, st0)
        got = np.array([a["dP_max"], a["avdP"], a["avbdP"], a["M0"]])
        assert np.all(np.abs(got - row_cq[1:]) <= 1e-15 * np.abs(row_cq[1:]) + 1e-19), (t, got, row_cq)
        assert abs(a["Pee"] - row_sp[1]) <= 5e-7 * abs(row_sp[1])
        assert abs(a["Pbee"] - row_sp[2]) <= 5e-7 * abs(row_sp[2])


def test_oracle_default_initial_condition(oracle):
    """NuOsc::initialize (src/initialize.hpp) through the fresh-start path."""
    case, d = load_golden("fv_default_ic")
    G, bG, st = oracle.init_reference(case, float(d["perturbation_size"]))
    inner = st[:, :, case.gz:case.gz + case.nz]
    assert np.array_equal(np.moveaxis(inner, 0, -1), d["state0"])  # bitwise
    assert np.array_equal(G[:, case.gz:case.gz + case.nz], d["G0"][..., 0])
    assert np.array_equal(bG[:, case.gz:case.gz + case.nz], d["G0"][..., 1])
    y = oracle.step(case, st, 10, coll_direct=True)
    assert _print_close(y[:, :, case.gz:case.gz + case.nz], d["rho_10"])
    # the t = 0 analysis row
    a = oracle.analyse(case, st, G, bG, st)
    cq0 = [ln for ln in text(d["conserved_quantities_txt"]).splitlines() if ln.startswith("0\t")][0]
    assert abs(float(cq0.split()[4]) - a["M0"]) <= 1e-15 * a["M0"]


def test_oracle_seeded_ic_hash(oracle):
    """The seeded initial condition is the one the fixtures were made from."""
    for name in ("c1_pre", "fv_small", "fd_small"):
        case, d = load_golden(name)
        G, bG, st = oracle.init_seeded(case, seed=int(d["seed"]))
        inner = np.ascontiguousarray(st[:, :, case.gz:case.gz + case.nz])
        assert hashlib.sha256(inner.tobytes()).hexdigest() == str(d["state0_sha256"])


def test_philox_known_answer(oracle):
    """Philox-4x32-10 known-answer vectors of the Random123 distribution
    (kat_vectors: philox4x32 10 rounds)."""
    assert list(oracle.philox([0, 0, 0, 0], [0, 0])) == \
        [0x6627e8d5, 0xe169c58d, 0xbc57ac4c, 0x9b00dbd8]
    assert list(oracle.philox([0xffffffff] * 4, [0xffffffff] * 2)) == \
        [0x408f276d, 0x41c83b0e, 0xa20bc7c6, 0x6d5451fd]
    assert list(oracle.philox([0x243f6a88, 0x85a308d3, 0x13198a2e, 0x03707344],
                              [0xa4093822, 0x299f31d0])) == \
        [0xd16cfe09, 0x94fdcceb, 0x5001e420, 0x24126ea1]


def _c1_run(oracle, name, nthreads=0):
    case, d = load_golden(name)
    G, bG, st0 = oracle.init_seeded(case, seed=int(d["seed"]))
    return case, d, G, bG, st0


def test_oracle_c1_pre_saturation(oracle):
    """The small FV workload as specified: 1024 x 64, 500 steps; subset, checksums and
    the analysis rows of the reference run."""
    case, d, G, bG, st0 = _c1_run(oracle, "c1_pre")
    y, t_prev = st0, 0
    for row in d["conserved_quantities"]:
        t = int(row[0])
        y = oracle.step(case, y, t - t_prev, nthreads=os.cpu_count() or 1)
        t_prev = t
        a = oracle.analyse(case, y, G, bG, st0)
        assert abs(a["M0"] - row[4]) <= 1e-12 * row[4]
        assert abs(a["dP_max"] - row[1]) <= 1e-9 * row[1] + 1e-18
    inner = y[:, :, case.gz:case.gz + case.nz]
    assert np.abs(inner[:, :, ::16] - d["rho_500_subset"]).max() <= 1e-13
    s = inner
    ck = np.stack([s.sum(axis=(1, 2)), (s * s).sum(axis=(1, 2)), np.abs(s).sum(axis=(1, 2))], 1)
    assert np.allclose(ck, d["rho_500_checksums"], rtol=1e-12, atol=1e-18)


@pytest.mark.slow
def test_oracle_c1_after_saturation(oracle):
    """The 1024 x 64 FV grid through saturation (1500 steps): survival
    probabilities and |M0| rows of the reference, <= 1e-6."""
    case, d, G, bG, st0 = _c1_run(oracle, "c1_sat")
    y, t_prev = st0, 0
    sp = d["survival_probability"]
    for row, row_sp in zip(d["conserved_quantities"], sp):
        t = int(row[0])
        y = oracle.step(case, y, t - t_prev, nthreads=os.cpu_count() or 1)
        t_prev = t
        a = oracle.analyse(case, y, G, bG, st0)
        assert abs(a["Pee"] - row_sp[1]) <= 1e-6
        assert abs(a["Pbee"] - row_sp[2]) <= 1e-6
        assert abs(a["M0"] - row[4]) <= 1e-6
        assert abs(a["dP_max"] - row[1]) <= 1e-6
    pee, pbee = oracle.pee_v(case, y, st0)
    assert np.abs(pee - d["rho_1500_pee_v"]).max() <= 1e-6
    assert np.abs(pbee - d["rho_1500_pbee_v"]).max() <= 1e-6


def test_oracle_fd_benchmark_grid_against_reference_run(oracle):
    """The oracle on the full FD benchmark grid (nz 32768 x nvz 256), 5 steps,
    against the reference's own dump: the stored columns to 1e-14 and the
    per-row checksums of the whole state to 1e-11 relative."""
    case, d = load_golden("c2_ref")
    G, bG, st0 = oracle.init_seeded(case, seed=int(d["seed"]))
    assert hashlib.sha256(st0[..., case.gz:case.gz + case.nz].tobytes()).hexdigest() == \
        str(d["state0_sha256"])
    s = oracle.step(case, st0, 5, nthreads=os.cpu_count() or 1)[..., case.gz:case.gz + case.nz]
    assert np.abs(s[:, :, d["columns"]] - d["rho_5_columns"]).max() <= 1e-14
    ck = np.stack([s.sum(axis=2), (s * s).sum(axis=2), np.abs(s).sum(axis=2)], -1)
    want = d["rho_5_row_checksums"]
    assert np.all(np.abs(ck - want) <= 1e-11 * np.abs(want) + 1e-13 * case.nz)

"""The drop-in driver (cosenu_b200/bin/cosenu_main) against the reference
driver's own outputs: same job.config / G0.bin / state0.bin in, the same
files out (src/main.cpp, src/snaps.hpp, src/analysis.hpp formats)."""
import os
import subprocess

import numpy as np
import pytest

from tests._util import load_golden, text, with_ghosts

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
DRIVER = os.path.join(ROOT, "cosenu_b200", "bin", "cosenu_main")


def _driver():
    if not os.path.exists(DRIVER):
        from cosenu_b200.build import build
        build()
    return DRIVER


def _write_presets(path, variant):
    from oracle.build import REF_VARIANTS
    with open(path, "w") as f:
        f.write("#if not defined(__PRESETS__)\n#define __PRESETS__\n\n")
        for m in REF_VARIANTS[variant]:
            f.write(f"#define {m}\n")
        f.write("\n#endif // __PRESETS__\n")


def _job(tmp_path, case, d, oracle, n_iter, anal, ndump):
    from oracle.oracle import job_config_dict, write_G0_bin, write_job_config, write_state_bin
    st0 = with_ghosts(case, d["state0"], oracle)
    G = with_ghosts(case, d["G"][None], oracle)[0]
    bG = with_ghosts(case, d["bG"][None], oracle)[0]
    write_job_config(str(tmp_path / "job.config"), job_config_dict(case, n_iter, anal, ndump))
    write_G0_bin(str(tmp_path / "G0.bin"), case, G, bG)
    write_state_bin(str(tmp_path / "state0.bin"), case, st0)
    _write_presets(str(tmp_path / "presets.hpp"), case.ref_variant())


def test_driver_rejects_incomplete_config(tmp_path):
    (tmp_path / "job.config").write_text("scheme : FV\nnz : 64\nbogus : 1\n")
    p = subprocess.run([_driver(), "--conf", "job.config"], cwd=tmp_path, capture_output=True,
                       text=True)
    assert p.returncode == 1
    assert "Redundant or unknown key: bogus" in p.stdout
    assert "[ FAIL ]...Incomplete config file" in p.stdout


def test_driver_requires_conf(tmp_path):
    p = subprocess.run([_driver()], cwd=tmp_path, capture_output=True, text=True)
    assert p.returncode == 1 and "--conf" in p.stdout


@pytest.mark.gpu
@pytest.mark.parametrize("name", ["fv_small", "fd_small", "fv_open", "fd_ko5"])
def test_driver_outputs_match_reference(tmp_path, oracle, name):
    case, d = load_golden(name)
    _job(tmp_path, case, d, oracle, int(d["n_iter"]), int(d["anal_every"]), int(d["n_dump_rho"]))
    p = subprocess.run([_driver(), "--conf", "job.config", "--ff", "--presets", "presets.hpp"],
                       cwd=tmp_path, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    from oracle.oracle import read_rho_dat, read_table
    for t in d["dump_steps"]:
        got = read_rho_dat(str(tmp_path / f"rho_{t}.dat"), case)
        assert np.abs(got - d[f"rho_{t}"]).max() <= 1e-10
    sp = read_table(str(tmp_path / "survival_probability.dat"))
    cq = read_table(str(tmp_path / "conserved_quantities.dat"))
    assert np.array_equal(sp[:, 0], d["survival_probability"][:, 0])
    assert np.abs(sp[:, 1:] - d["survival_probability"][:, 1:]).max() <= 5e-7
    assert np.array_equal(cq[:, 0], d["conserved_quantities"][:, 0])
    assert np.all(np.abs(cq[:, 1:] - d["conserved_quantities"][:, 1:])
                  <= 1e-12 * np.maximum(np.abs(d["conserved_quantities"][:, 1:]), 1.0))
    if "rho_first_txt" in d:
        # text layout: identical line structure and identical Z / vz columns
        ref_lines = text(d["rho_first_txt"]).split("\n")
        got_lines = open(tmp_path / f"rho_{int(d['dump_steps'][0])}.dat").read().split("\n")
        assert len(ref_lines) == len(got_lines)
        for a, b in zip(ref_lines, got_lines):
            assert a.split("\t")[:2] == b.split("\t")[:2]


@pytest.mark.gpu
def test_driver_fresh_start_matches_reference(tmp_path):
    """No --ff: the reference's initialize() path, G0.bin / state0.bin bytes
    and the t = 0 snapshot text byte for byte."""
    import json
    from oracle.oracle import job_config_dict, write_job_config, Case
    case, d = load_golden("fv_default_ic")
    write_job_config(str(tmp_path / "job.config"),
                     job_config_dict(case, 11, 5, 2, float(d["perturbation_size"])))
    p = subprocess.run([_driver(), "--conf", "job.config"], cwd=tmp_path, capture_output=True,
                       text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    g0 = np.fromfile(tmp_path / "G0.bin", "<f8").reshape(case.nvz, case.nz, 2)
    s0 = np.fromfile(tmp_path / "state0.bin", "<f8").reshape(case.nvz, case.nz, 8)
    assert np.array_equal(g0, d["G0"])
    assert np.array_equal(s0, d["state0"])
    assert open(tmp_path / "rho_0.dat").read() == text(d["rho_0_txt"])
    sp_ref = text(d["survival_probability_txt"]).splitlines()
    sp_got = open(tmp_path / "survival_probability.dat").read().splitlines()
    assert sp_got[:2] == sp_ref[:2]  # header and the t = 0 row
    cq_ref = text(d["conserved_quantities_txt"]).splitlines()
    cq_got = open(tmp_path / "conserved_quantities.dat").read().splitlines()
    assert cq_got[0] == cq_ref[0]
    assert len(cq_got) == len(cq_ref)


@pytest.mark.gpu
def test_driver_checkpoint_and_resume(tmp_path, oracle):
    """--checkpoint-every writes state.bin (src/snaps.hpp:6-39 format) from
    the asynchronous device snapshot while stepping goes on; its header is
    the next iteration to run, so a run resumed from it with --ff ends where
    the uninterrupted reference run ends."""
    import shutil
    from oracle.oracle import read_rho_dat, read_state_bin
    case, d = load_golden("fv_small")
    n_iter, anal, ndump = int(d["n_iter"]), int(d["anal_every"]), int(d["n_dump_rho"])
    a = tmp_path / "a"
    a.mkdir()
    _job(a, case, d, oracle, n_iter, anal, ndump)
    p = subprocess.run([_driver(), "--conf", "job.config", "--ff", "--presets", "presets.hpp",
                        "--checkpoint-every", "15"], cwd=a, capture_output=True, text=True,
                       timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    st, t = read_state_bin(str(a / "state.bin"), case, header=True)
    assert t == 16
    assert np.abs(st[:, :, case.gz:case.gz + case.nz] - d["rho_15"]).max() <= 1e-10
    assert not any(f.startswith("state1") for f in os.listdir(a))  # renamed into place
    b = tmp_path / "b"
    b.mkdir()
    for f in ("job.config", "G0.bin", "state0.bin", "presets.hpp", "state.bin"):
        shutil.copy(a / f, b / f)
    p = subprocess.run([_driver(), "--conf", "job.config", "--ff", "--presets", "presets.hpp"],
                       cwd=b, capture_output=True, text=True, timeout=300)
    assert p.returncode == 0, p.stdout + p.stderr
    assert "Starting time = 16" in p.stdout
    got = read_rho_dat(str(b / "rho_20.dat"), case)
    assert np.abs(got - d["rho_20"]).max() <= 1e-10
    assert not (b / "rho_15.dat").exists()

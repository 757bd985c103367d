"""The drop-in driver's input parsers (include/cosenu_nuosc.hpp) on the CPU:
job.config keys as manage.py writes them (src/parser.hpp:46-256) and the
presets.hpp switches (manage.py:160-186), for every switch combination the
reference binaries were built with; the dump cadence agrees with the
snapshots the reference itself wrote."""
import json
import os
import subprocess

import numpy as np
import pytest

from tests._util import load_golden

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def parse_bin(tmp_path_factory):
    from cosenu_b200 import _lib
    if not os.path.exists(_lib.LIB_PATH):
        from cosenu_b200.build import build
        build()
    lib_dir = os.path.dirname(_lib.LIB_PATH)
    out = tmp_path_factory.mktemp("parse") / "parse_main"
    subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "native", "parse_main.cpp"), "-o", str(out),
                    "-L", lib_dir, "-lcosenu_b200", f"-Wl,-rpath,{lib_dir}"], check=True)
    return str(out)


def _parse(parse_bin, tmp_path, d, variant, need_vac=True, need_coll=True):
    from oracle.build import REF_VARIANTS
    from oracle.oracle import write_job_config
    write_job_config(str(tmp_path / "job.config"), d)
    with open(tmp_path / "presets.hpp", "w") as f:
        f.write("#if not defined(__PRESETS__)\n#define __PRESETS__\n\n")
        for m in REF_VARIANTS[variant]:
            f.write(f"#define {m}\n")
        f.write("\n#endif // __PRESETS__\n")
    p = subprocess.run([parse_bin, str(tmp_path / "job.config"), str(tmp_path / "presets.hpp"),
                        str(int(need_vac)), str(int(need_coll))], capture_output=True, text=True,
                       check=True)
    return json.loads(p.stdout)


@pytest.mark.parametrize("name", ["fv_small", "fd_small", "fv_open", "fd_open", "fv_mat",
                                  "fd_mat", "fd_ko5", "fv_advoff", "fd_advoff"])
def test_parsers_read_what_the_reference_reads(parse_bin, tmp_path, name):
    from oracle.oracle import job_config_dict
    case, g = load_golden(name)
    d = job_config_dict(case, int(g["n_iter"]), int(g["anal_every"]), int(g["n_dump_rho"]))
    r = _parse(parse_bin, tmp_path, d, case.ref_variant())
    assert r["error"] == "" and r["p_error"] == ""
    for k in ("N_ITER", "ANAL_EVERY", "nz", "nvz", "gz", "z0", "z1", "v0", "v1", "CFL", "pmo",
              "omega", "theta", "mu"):
        assert r[k] == d[k], k
    # the reference dumped at multiples of its dump interval
    steps = [int(t) for t in g["dump_steps"]]
    assert all(t % r["dump_interval"] == 0 for t in steps)
    assert steps == [t for t in range(1, int(g["n_iter"])) if t % r["dump_interval"] == 0]
    # switches: scheme, boundary, FD variant, physics terms
    assert r["p_scheme"] == (1 if case.scheme == "fd" else 0)
    assert r["p_bc"] == (1 if case.bc == "open" else 0)
    if case.scheme == "fd":
        assert r["p_fd_advec"] == 0 and r["p_ko_order"] == case.ko_order
    flags = r["p_flags"]
    assert bool(flags & 1) == case.vac and bool(flags & 4) == case.coll
    assert bool(flags & 2) == case.mat and bool(flags & 8) == case.advec_off


def test_incomplete_config_reports_the_reference_message(parse_bin, tmp_path):
    from oracle.oracle import job_config_dict
    case, g = load_golden("fv_small")
    d = job_config_dict(case, 21, 5, 4)
    del d["mu"]
    r = _parse(parse_bin, tmp_path, d, "fv", need_coll=True)
    assert "Incomplete config file" in r["error"]
    r = _parse(parse_bin, tmp_path, d, "fv", need_coll=False)  # mu only needed with COLL_OSC_ON
    assert r["error"] == ""

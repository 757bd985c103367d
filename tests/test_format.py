"""The multi-threaded rho_<t>.dat writer (include/cosenu_format.hpp) on the
CPU: byte-identical to the text the reference's dump_rho wrote
(src/snaps.hpp:187-218) for the same state, whatever the thread count."""
import os
import subprocess

import numpy as np
import pytest

from tests._util import load_golden, text

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.fixture(scope="module")
def format_bin(tmp_path_factory):
    out = tmp_path_factory.mktemp("fmt") / "format_rho_main"
    subprocess.run(["g++", "-std=c++17", "-O2", "-pthread", "-I", os.path.join(ROOT, "include"),
                    os.path.join(ROOT, "tests", "native", "format_rho_main.cpp"), "-o", str(out)],
                   check=True)
    return str(out)


def _grid(case):
    # NuOsc constructor (src/nuosc.hpp:83-92)
    Z = np.array([case.z0 + (j + 0.5) * case.dz for j in range(case.nz)])
    vz = np.array([case.v0 + (i + 0.5) * case.dv for i in range(case.nvz)])
    return Z, vz


def _format(format_bin, tmp_path, case, state, nthreads):
    Z, vz = _grid(case)
    src = tmp_path / f"in_{nthreads}.bin"
    with open(src, "wb") as f:
        np.array([case.nz, case.nvz, nthreads], dtype="<i4").tofile(f)
        Z.astype("<f8").tofile(f)
        vz.astype("<f8").tofile(f)
        np.ascontiguousarray(state, dtype="<f8").tofile(f)
    dst = tmp_path / f"rho_{nthreads}.dat"
    subprocess.run([format_bin, str(src), str(dst)], check=True)
    return open(dst, "rb").read()


@pytest.mark.parametrize("nthreads", [1, 3, 8])
def test_rho_text_matches_reference(format_bin, tmp_path, nthreads):
    case, d = load_golden("fv_default_ic")
    state = np.moveaxis(d["state0"], 2, 0)          # [nvz][nz][8] -> [8][nvz][nz]
    got = _format(format_bin, tmp_path, case, state, nthreads)
    assert got == text(d["rho_0_txt"]).encode()


def test_rho_text_special_values(format_bin, tmp_path):
    """Zeros of either sign, integers and values whose 16-digit form needs an
    exponent print as the iostream writer prints them."""
    case, _ = load_golden("fv_default_ic")
    rng = np.random.default_rng(5)
    state = (rng.standard_normal((8, case.nvz, case.nz)) *
             10.0 ** rng.integers(-30, 30, (8, case.nvz, case.nz)))
    state[:4, 0, 0] = [0.0, -0.0, 1.0, -1e-300]
    lines = _format(format_bin, tmp_path, case, state, 4).decode().split("\n")
    Z, vz = _grid(case)
    first = lines[0].split("\t")
    assert first[:2] == ["%.6g" % Z[0], "%.6g" % vz[0]]
    assert first[2:6] == ["0", "-0", "1", "-1e-300"]
    v = lines[1].split("\t")
    assert v[0] == "%.16g" % Z[0] and v[1] == "%.16g" % vz[1]
    assert v[2:10] == ["%.16g" % state[c, 1, 0] for c in range(8)]

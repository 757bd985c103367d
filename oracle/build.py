"""Build recipe for the oracle side (test infrastructure only).

1. ``oracle/libcosenu_oracle.so`` -- the plain-C restatement in
   ``cosenu_oracle.c`` (gcc, -O3, no FMA contraction, no fast-math, so its
   arithmetic rounds like the reference build).
2. ``oracle/_ref/cosenu_ref_<variant>`` -- the reference's own driver
   (``src/main.cpp`` of COSEnu) compiled straight from its source tree with the
   reference's ``--mcore`` flags (manage.py:29-31,305-306:
   ``g++ -std=c++0x -O3 -fopenmp``).  The compile-time switches that
   manage.py would write into ``src/presets.hpp`` (manage.py:160-186) are
   supplied instead through a forced include written into ``oracle/_ref/``
   that also defines the header guard, so the checked-in presets file is
   skipped and nothing in the reference tree is modified or copied.

Step 2 runs only where the reference tree exists (the development container);
elsewhere the binaries already built travel with the repository snapshot.
"""
from __future__ import annotations

import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
# the COSEnu source tree: COSENU_REFERENCE_ROOT, else a "reference" directory
# beside this repository's checkout
REF_ROOT = os.environ.get("COSENU_REFERENCE_ROOT") or os.path.join(
    os.path.dirname(os.path.dirname(HERE)), "reference")
REF_OUT = os.path.join(HERE, "_ref")
ORACLE_SO = os.path.join(HERE, "libcosenu_oracle.so")

# variant name -> preset macros (the same sets manage.py:160-186 emits)
REF_VARIANTS = {
    "fv": ["PERIODIC_BC", "FV", "VAC_OSC_ON", "COLL_OSC_ON"],
    "fd": ["PERIODIC_BC", "FD", "KO_ORD_3", "ADVEC_CENTER_FD", "VAC_OSC_ON", "COLL_OSC_ON"],
    "fv_open": ["OPEN_BC", "FV", "VAC_OSC_ON", "COLL_OSC_ON"],
    "fd_open": ["OPEN_BC", "FD", "KO_ORD_3", "ADVEC_CENTER_FD", "VAC_OSC_ON", "COLL_OSC_ON"],
    "fv_mat": ["PERIODIC_BC", "FV", "VAC_OSC_ON", "MAT_OSC_ON", "COLL_OSC_ON"],
    "fd_mat": ["PERIODIC_BC", "FD", "KO_ORD_3", "ADVEC_CENTER_FD", "VAC_OSC_ON", "MAT_OSC_ON",
               "COLL_OSC_ON"],
    "fd_ko5": ["PERIODIC_BC", "FD", "ADVEC_CENTER_FD", "VAC_OSC_ON", "COLL_OSC_ON"],
    "fv_advoff": ["PERIODIC_BC", "FV", "VAC_OSC_ON", "COLL_OSC_ON", "ADVEC_OFF"],
    "fd_advoff": ["PERIODIC_BC", "FD", "KO_ORD_3", "ADVEC_CENTER_FD", "VAC_OSC_ON", "COLL_OSC_ON",
                  "ADVEC_OFF"],
}


def _newer(target: str, *sources: str) -> bool:
    if not os.path.exists(target):
        return False
    t = os.path.getmtime(target)
    return all(os.path.getmtime(s) <= t for s in sources if os.path.exists(s))


def build_oracle(force: bool = False) -> str:
    src = os.path.join(HERE, "cosenu_oracle.c")
    if force or not _newer(ORACLE_SO, src):
        cmd = ["gcc", "-O3", "-std=c99", "-D_GNU_SOURCE", "-ffp-contract=off", "-fopenmp",
               "-shared", "-fPIC", src, "-o", ORACLE_SO + ".tmp", "-lm"]
        subprocess.run(cmd, check=True)
        os.replace(ORACLE_SO + ".tmp", ORACLE_SO)
    return ORACLE_SO


def reference_available() -> bool:
    return os.path.isfile(os.path.join(REF_ROOT, "src", "main.cpp"))


def ref_binary(variant: str) -> str:
    return os.path.join(REF_OUT, f"cosenu_ref_{variant}")


def _build_one(variant: str, macros: list[str], force: bool) -> str:
    exe = ref_binary(variant)
    main = os.path.join(REF_ROOT, "src", "main.cpp")
    hdrs = [os.path.join(REF_ROOT, "src", f) for f in os.listdir(os.path.join(REF_ROOT, "src"))]
    if not force and _newer(exe, main, *hdrs, __file__):
        return exe
    preset = os.path.join(REF_OUT, f"presets_{variant}.hpp")
    with open(preset, "w") as f:
        f.write("/* forced include: compile-time switches for one reference variant */\n")
        f.write("#define __PRESETS__\n")
        for m in macros:
            f.write(f"#define {m}\n")
    cmd = ["g++", "-std=c++0x", "-O3", "-fopenmp", "-include", preset, main, "-o", exe + ".tmp"]
    subprocess.run(cmd, check=True, capture_output=True)
    os.replace(exe + ".tmp", exe)
    return exe


def build_reference(force: bool = False) -> dict[str, str]:
    """Compile every reference variant; returns {} when the tree is absent."""
    if not reference_available():
        return {}
    if shutil.which("g++") is None:
        raise RuntimeError("g++ not found; cannot compile the reference")
    os.makedirs(REF_OUT, exist_ok=True)
    out = {}
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        futs = {ex.submit(_build_one, v, m, force): v for v, m in REF_VARIANTS.items()}
        for fut in cf.as_completed(futs):
            out[futs[fut]] = fut.result()
    return out


def build(force: bool = False) -> None:
    build_oracle(force)
    if not reference_available():
        print(f"oracle/build.py: no COSEnu tree at {REF_ROOT} (set COSENU_REFERENCE_ROOT); "
              "reference binaries not rebuilt", file=sys.stderr)
        return
    build_reference(force)


if __name__ == "__main__":
    build(force="--force" in sys.argv)
    print("oracle:", ORACLE_SO)
    for v in REF_VARIANTS:
        p = ref_binary(v)
        print(f"ref[{v}]:", p if os.path.exists(p) else "(not built)")

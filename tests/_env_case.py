"""Runs small reference fixtures through the TMA-pipelined kernel in a fresh
process, so that tuning switches read once per process (COSENU_TMA_MINB,
COSENU_TMA_RING) take effect; prints the largest deviation from the
reference's snapshots and exits non-zero above 1e-10.
Usage: python -m tests._env_case <fixture> [<fixture> ...]"""
import json
import os
import sys

import numpy as np

from oracle.oracle import Oracle
from tests._util import gpu_from_case, load_golden, with_ghosts


def main(names):
    os.environ["COSENU_KERNEL"] = "tma"
    oracle = Oracle()
    worst = {}
    for name in names:
        case, d = load_golden(name)
        st0 = with_ghosts(case, d["state0"], oracle)
        with gpu_from_case(case) as sim:
            sim.upload(st0)
            t_prev, err = 0, 0.0
            for t in d["dump_steps"]:
                sim.evolve(int(t) - t_prev)
                t_prev = int(t)
                got = sim.download()[..., case.gz:case.gz + case.nz]
                err = max(err, float(np.abs(got - d[f"rho_{t}"]).max()))
        worst[name] = err
    print(json.dumps(worst))
    return 0 if max(worst.values()) <= 1e-10 else 1


if __name__ == "__main__":
    sys.exit(main(sys.argv[1:]))

"""Ensembles (cosenu_batch_*): members of uneven nz / nvz / physics and step
counts advanced by shared stage launches must match the same simulations
run one at a time (and the oracle)."""
import math
import os

import numpy as np
import pytest

from cosenu_b200.ensemble import Instance, ensemble_instances, steps_to


def test_ensemble_instance_distribution():
    xs = ensemble_instances(256)
    nz = np.array([x.nz for x in xs])
    assert len(xs) == 256
    assert nz.min() >= 512 and nz.max() <= 8192 and np.all(nz % 256 == 0)
    assert set(x.nvz for x in xs) == {32, 64, 128, 256}
    for x in xs:
        assert 0.6 <= x.alpha <= 1.2 and 0.4 <= x.sig_nu <= 0.8 and 0.3 <= x.sig_nubar <= 0.7
        assert 0.5 <= x.mu <= 2.0
        dt = 0.4 * 1200.0 / x.nz
        assert (x.nsteps - 1) * dt < 1000.0 / x.mu <= x.nsteps * dt + 1e-9
    # deterministic
    assert [x.nz for x in ensemble_instances(256)] == list(nz)
    assert steps_to(10.0, 1200) == 25


def _small(seed=3):
    rng = np.random.default_rng(seed)
    out = []
    for i, (nz, nvz) in enumerate([(256, 32), (512, 24), (1024, 64), (256, 8), (768, 40),
                                   (4736, 16)]):
        out.append(Instance(nz=nz, nvz=nvz, alpha=float(rng.uniform(0.6, 1.2)),
                            sig_nu=float(rng.uniform(0.4, 0.8)),
                            sig_nubar=float(rng.uniform(0.3, 0.7)),
                            mu=float(rng.uniform(0.5, 2.0)), seed=100 + i,
                            nsteps=int(rng.integers(5, 40)), z0=-nz / 2, z1=nz / 2))
    return out


def _standalone(x, i, scheme, precision, **kw):
    from cosenu_b200 import NuOsc
    sim = NuOsc(nz=x.nz, nvz=x.nvz, gz=4, z0=x.z0, z1=x.z1, cfl=x.cfl, omega=0.0, mu=x.mu,
                scheme=scheme, precision=precision, **kw)
    sim.init_seeded(x.seed, instance=i, sig_nu=x.sig_nu, sig_nubar=x.sig_nubar, alpha=x.alpha)
    sim.evolve(x.nsteps)
    out = sim.download()
    sim.close()
    return out


@pytest.mark.gpu
@pytest.mark.parametrize("precision", ["fp64", "fp32"])
@pytest.mark.parametrize("scheme", ["fv", "fd"])
def test_ensemble_tma_matches_members_run_alone(gpu_lib, monkeypatch, scheme, precision):
    """FP32-bulk members alternate their two state buffers every step, so the
    ensemble launches use per-parity argument and tensor-map sets: odd and even
    step counts (5..39) and phases of both parities are covered."""
    from cosenu_b200.ensemble import Ensemble
    xs = _small()
    monkeypatch.setenv("COSENU_KERNEL", "tma")  # standalone runs use the same kernel family
    with Ensemble(xs, scheme=scheme, precision=precision) as ens:
        assert ens.config()["use_tma"]
        ens.init_seeded()
        ens.run()
        ens.synchronize()
        for i, (x, m) in enumerate(zip(xs, ens.members)):
            assert m.steps == x.nsteps
            got = m.download()
            want = _standalone(x, i, scheme, precision)
            assert np.abs(got - want).max() <= 1e-13, i


@pytest.mark.gpu
@pytest.mark.parametrize("tz", [32, 16, 8])
def test_ensemble_register_tiled_matches_members(gpu_lib, oracle, tz):
    from cosenu_b200.ensemble import Ensemble
    xs = _small()
    tvs = [8, 24, 16, 8, 40, 16]
    with Ensemble(xs, scheme="fv") as ens:
        ens.set_config(False, tz, tvs)
        ens.init_seeded()
        ens.run()
        ens.synchronize()
        for i, (x, m) in enumerate(zip(xs, ens.members)):
            got = m.download()
            want = _standalone(x, i, "fv", "fp64", tile_z=tz, tile_v=tvs[i])
            assert np.abs(got - want).max() <= 1e-13, i
        # one member against the CPU oracle
        from oracle.oracle import Case
        x = xs[1]
        case = Case(nz=x.nz, nvz=x.nvz, gz=4, z0=x.z0, z1=x.z1, scheme="fv", omega=0.0, mu=x.mu)
        G, bG, st0 = oracle.init_seeded(case, seed=x.seed, instance=1, sig_nu=x.sig_nu,
                                        sig_nubar=x.sig_nubar, alpha=x.alpha)
        ref = oracle.step(case, st0, x.nsteps)
        assert np.abs(ens.members[1].download() - ref).max() <= 1e-12


@pytest.mark.gpu
def test_ensemble_autotune_keeps_results(gpu_lib):
    from cosenu_b200.ensemble import Ensemble
    xs = _small()
    with Ensemble(xs) as ens:
        ens.init_seeded()
        before = [m.download() for m in ens.members]
        report = ens.autotune(trial_steps=2)
        assert "chosen:" in report
        # states and step counters restored
        for m, b in zip(ens.members, before):
            assert m.steps == 0
            assert np.array_equal(m.download(), b)
        ens.run()
        ens.synchronize()
        cfg = ens.config()
        for i, (x, m) in enumerate(zip(xs, ens.members)):
            kw = {} if cfg["use_tma"] else {"tile_z": cfg["tz"], "tile_v": cfg["tv"][i]}
            if cfg["use_tma"]:
                os.environ["COSENU_KERNEL"] = "tma"
            try:
                want = _standalone(x, i, "fv", "fp64", **kw)
            finally:
                os.environ.pop("COSENU_KERNEL", None)
            assert np.abs(m.download() - want).max() <= 1e-13, i


@pytest.mark.gpu
def test_ensemble_fp32_bulk_close_to_fp64(gpu_lib):
    from cosenu_b200.ensemble import Ensemble
    xs = _small()
    outs = []
    for prec in ("fp64", "fp32"):
        with Ensemble(xs, precision=prec) as ens:
            ens.init_seeded()
            ens.run()
            ens.synchronize()
            outs.append([m.download() for m in ens.members])
    # 5-40 steps before saturation: the increment form stays within 1e-9 of FP64
    for a, b in zip(*outs):
        assert np.abs(a - b).max() <= 1e-9


@pytest.mark.gpu
def test_sharded_runner_on_one_gpu_matches_members_run_alone(gpu_lib):
    """run_ensemble_sharded on one process (the path bench.py's ensemble
    workload takes at every N): autotuned ensemble, every member's final
    analysis equal to the member run alone to 1e-12."""
    import dataclasses

    from cosenu_b200 import NuOsc
    from cosenu_b200.distributed import run_ensemble_sharded
    xs = [dataclasses.replace(x, index=i) for i, x in enumerate(_small())]
    res, secs, share = run_ensemble_sharded(xs, None, trial_steps=1)
    assert share == list(range(len(xs))) and secs > 0
    for i, x in enumerate(xs):
        sim = NuOsc(nz=x.nz, nvz=x.nvz, gz=4, z0=x.z0, z1=x.z1, cfl=x.cfl, omega=0.0, mu=x.mu,
                    scheme="fv")
        sim.init_seeded(x.seed, instance=i, sig_nu=x.sig_nu, sig_nubar=x.sig_nubar,
                        alpha=x.alpha)
        sim.evolve(x.nsteps)
        a = sim.analyse()
        sim.close()
        for k in ("Pee", "Pbee", "M0", "trace", "eln"):
            assert abs(a[k] - res[i][k]) <= 1e-12 * max(1.0, abs(a[k])), (i, k)

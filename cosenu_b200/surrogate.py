"""Learned surrogate for the late-time angle-resolved survival probability.

Input: the initial nu and nubar angular profiles G(v), bG(v) on the solver's
velocity grid plus (alpha, mu).  Output: P_ee(v) = sum_z ee / sum_z ee0 per
velocity bin (the per-v analogue of surv_prob, src/analysis.hpp:169-176),
averaged over the final 20 % of a run to t = t_factor / mu.  Training data come
from the ensemble solver (cosenu_b200.ensemble); the network is trained on the
GPU by the library's own kernels (cosenu_mlp_*).  A few networks trained from
different initialisations form a committee; where they disagree by more than
a threshold the prediction is not trusted and the solver is run instead.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .ensemble import Ensemble, Instance, steps_to


def gauss_profile(v: np.ndarray, v0: float, sigma: float) -> np.ndarray:
    """Normalised Gaussian angular profile on [-1, 1]
    (src/miscellaneous_funcs.hpp:57-62)."""
    e = (v - v0) ** 2 / (2.0 * sigma * sigma)
    N = sigma * math.sqrt(math.pi / 2.0) * (math.erf((1.0 + v0) / sigma / math.sqrt(2.0)) +
                                            math.erf((1.0 - v0) / sigma / math.sqrt(2.0)))
    return np.exp(-e) / N


def features(x: Instance) -> np.ndarray:
    v = -1.0 + (np.arange(x.nvz) + 0.5) * (2.0 / x.nvz)
    return np.concatenate([gauss_profile(v, 1.0, x.sig_nu),
                           x.alpha * gauss_profile(v, 1.0, x.sig_nubar),
                           [x.alpha, x.mu]]).astype(np.float32)


def reseeded(instances: list[Instance], offset: int = 7919) -> list[Instance]:
    """The same physical set-ups with different random perturbations (the
    seed-to-seed spread of the solver is the noise floor of any predictor of
    P_ee(v) from the angular profiles alone)."""
    import dataclasses
    return [dataclasses.replace(x, seed=x.seed + offset) for x in instances]


def surrogate_instances(n: int, seed: int, nz: int | None = 512, nvz: int = 128,
                        t_factor: float = 1000.0, nz_range=(512, 8192)) -> list[Instance]:
    """Surrogate inputs: the ensemble parameter distribution
    (ensemble.ensemble_instances) at fixed nvz, with nz fixed (to keep a
    training set affordable) or, with nz=None, log-uniform in nz_range rounded
    to 256 as in the ensemble workload."""
    rng = np.random.default_rng(seed)
    out = []
    for i in range(n):
        mu = float(rng.uniform(0.5, 2.0))
        if nz is None:
            lo, hi = math.log(nz_range[0]), math.log(nz_range[1])
            nzi = int(256 * round(math.exp(rng.uniform(lo, hi)) / 256))
            nzi = min(max(nzi, 256), nz_range[1])
        else:
            nzi = nz
        out.append(Instance(nz=nzi, nvz=nvz, alpha=float(rng.uniform(0.6, 1.2)),
                            sig_nu=float(rng.uniform(0.4, 0.8)),
                            sig_nubar=float(rng.uniform(0.3, 0.7)), mu=mu,
                            seed=seed * 100000 + i, nsteps=steps_to(t_factor / mu, nzi)))
    return out


def solve_pee(instances: list[Instance], chunk: int = 256, samples: int = 20,
              tail: float = 0.2, stream=None) -> np.ndarray:
    """Ensemble-solver targets: P_ee(v) averaged over `samples` equally spaced
    times in the last `tail` of each run; returns [n][nvz]."""
    out = np.zeros((len(instances), instances[0].nvz))
    for c0 in range(0, len(instances), chunk):
        xs = instances[c0:c0 + chunk]
        with Ensemble(xs) as ens:
            if stream is not None:
                ens.set_stream(stream)
            ens.init_seeded()
            n = np.array([x.nsteps for x in xs])
            start = np.floor(n * (1.0 - tail)).astype(int)
            marks = [start + np.round((n - start) * (k + 1) / samples).astype(int)
                     for k in range(samples)]
            done = np.zeros_like(n)
            acc = np.zeros((len(xs), xs[0].nvz))
            for target in [start] + marks:
                ens.run((target - done).tolist())
                done = target
                if target is start:
                    continue
                ens.synchronize()
                for i, m in enumerate(ens.members):
                    acc[i] += m.pee_v()[0]
            out[c0:c0 + len(xs)] = acc / samples
    return out


class MLP:
    """The library's surrogate network (cosenu_mlp_*)."""

    def __init__(self, n_in: int = 258, n_hidden: int = 512, n_layers: int = 3, n_out: int = 128,
                 seed: int = 0, device: int = 0):
        self.lib = L.load()
        h = C.c_void_p()
        rc = self.lib.cosenu_mlp_create(n_in, n_hidden, n_layers, n_out, seed, device,
                                        C.byref(h))
        if rc != L.OK:
            raise L.CosenuError(rc, "cosenu_mlp_create failed")
        self.h = h
        self.n_in, self.n_out = n_in, n_out
        n = C.c_size_t()
        self.lib.cosenu_mlp_num_params(self.h, C.byref(n))
        self.nparam = n.value

    def _check(self, rc):
        if rc != L.OK:
            raise L.CosenuError(rc, self.lib.cosenu_mlp_last_error(self.h).decode())

    def close(self):
        if getattr(self, "h", None):
            self.lib.cosenu_mlp_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def params(self) -> np.ndarray:
        p = np.zeros(self.nparam, dtype=np.float32)
        self._check(self.lib.cosenu_mlp_get_params(self.h, p.ctypes.data))
        return p

    def set_params(self, p: np.ndarray) -> None:
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self.lib.cosenu_mlp_set_params(self.h, p.ctypes.data))

    def forward(self, x: np.ndarray) -> np.ndarray:
        x = np.ascontiguousarray(x, dtype=np.float32)
        y = np.zeros((x.shape[0], self.n_out), dtype=np.float32)
        self._check(self.lib.cosenu_mlp_forward(self.h, x.ctypes.data, x.shape[0], y.ctypes.data))
        return y

    def loss_grad(self, x: np.ndarray, t: np.ndarray):
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        g = np.zeros(self.nparam, dtype=np.float32)
        loss = C.c_float()
        self._check(self.lib.cosenu_mlp_loss_grad(self.h, x.ctypes.data, t.ctypes.data,
                                                  x.shape[0], C.byref(loss), g.ctypes.data))
        return loss.value, g

    def set_data(self, x: np.ndarray, t: np.ndarray) -> None:
        """Training set, held on the device for train()."""
        x = np.ascontiguousarray(x, dtype=np.float32)
        t = np.ascontiguousarray(t, dtype=np.float32)
        self._check(self.lib.cosenu_mlp_set_data(self.h, x.ctypes.data, t.ctypes.data,
                                                 x.shape[0]))

    def train(self, epochs: int = 200, batch: int = 256, lr: float = 1e-3,
              weight_decay: float = 1e-4, seed: int = 0) -> np.ndarray:
        """AdamW epochs over the data of set_data(); returns each epoch's mean loss."""
        losses = np.zeros(epochs, dtype=np.float32)
        self._check(self.lib.cosenu_mlp_train(self.h, epochs, batch, lr, weight_decay, 0.9, 0.999,
                                              1e-8, seed, losses.ctypes.data))
        return losses

    def fit(self, x: np.ndarray, t: np.ndarray, epochs: int = 200, batch: int = 256,
            lr: float = 1e-3, weight_decay: float = 1e-4, seed: int = 0) -> np.ndarray:
        self.set_data(x, t)
        return self.train(epochs, batch, lr, weight_decay, seed)

    def set_timing(self, on: bool) -> None:
        """CUDA-event timing of every later launch by kernel class (clears the totals)."""
        self._check(self.lib.cosenu_mlp_set_timing(self.h, int(on)))

    def timing(self) -> dict:
        """Device milliseconds per kernel class since set_timing(True)."""
        ms = (C.c_double * 3)()
        self._check(self.lib.cosenu_mlp_timing(self.h, ms))
        return {"gemm": ms[0], "elementwise": ms[1], "adamw": ms[2]}


@dataclass
class Prediction:
    pee: np.ndarray          # [n][nvz] final answer
    spread: np.ndarray       # [n] RMS over v of the committee's standard deviation
    fallback: np.ndarray     # [n] bool: solver used


class Surrogate:
    """Committee of networks with solver fallback.  Inputs are standardised
    per feature with the training set's mean and spread."""

    def __init__(self, n_models: int = 4, **mlp_kw):
        self.models = [MLP(seed=1000 + k, **mlp_kw) for k in range(n_models)]
        self.x_mean = None
        self.x_std = None

    def _norm(self, x) -> np.ndarray:
        x = np.asarray(x, dtype=np.float64)
        if self.x_mean is None:
            return x.astype(np.float32)
        return ((x - self.x_mean) / self.x_std).astype(np.float32)

    def fit(self, x, t, epochs: int = 300, lr: float = 2e-3, schedule="cos",
            **kw) -> list[np.ndarray]:
        """AdamW from the library's training kernels.  schedule "cos": the
        learning rate follows lr * (1 + cos(pi e / epochs)) / 2 over the epochs;
        a tuple of factors: equal segments of the epochs at lr * factor.  The
        optimizer state carries over between epochs and segments."""
        x = np.asarray(x, dtype=np.float64)
        self.x_mean = x.mean(axis=0)
        self.x_std = x.std(axis=0) + 1e-6
        xn = self._norm(x)
        if schedule == "cos":
            plan = [(1, 0.5 * (1.0 + math.cos(math.pi * e / epochs))) for e in range(epochs)]
        else:
            seg = max(1, epochs // len(schedule))
            plan = [(seg, f) for f in schedule]
        out = []
        for k, m in enumerate(self.models):
            m.set_data(xn, t)
            out.append(np.concatenate([m.train(epochs=n, lr=lr * f, seed=k + 1 + 100 * j, **kw)
                                       for j, (n, f) in enumerate(plan)]))
        return out

    def committee(self, x) -> tuple[np.ndarray, np.ndarray]:
        """Committee mean and disagreement (RMS over v of the members' standard
        deviation) per instance."""
        xn = self._norm(x)
        ys = np.stack([m.forward(xn) for m in self.models])
        return ys.mean(axis=0), np.sqrt((ys.std(axis=0) ** 2).mean(axis=1))

    def predict(self, instances: list[Instance], threshold: float = 1e-2,
                solver=solve_pee) -> Prediction:
        x = np.stack([features(i) for i in instances])
        mean, spread = self.committee(x)
        fb = spread > threshold
        pee = mean.astype(np.float64)
        if fb.any():
            idx = np.nonzero(fb)[0]
            pee[idx] = solver([instances[i] for i in idx])
        return Prediction(pee=pee, spread=spread, fallback=fb)

    def set_timing(self, on: bool) -> None:
        for m in self.models:
            m.set_timing(on)

    def timing(self) -> dict:
        """Device milliseconds per kernel class, summed over the committee."""
        out = {"gemm": 0.0, "elementwise": 0.0, "adamw": 0.0}
        for m in self.models:
            for k, v in m.timing().items():
                out[k] += v
        return out

    def close(self):
        for m in self.models:
            m.close()

"""Surrogate network kernels (cosenu_mlp_*) against the FP64 CPU oracle
(oracle/mlp_oracle.py): the oracle's own analytic gradient against central
finite differences, then the GPU forward pass and gradients against the
oracle with the BF16 rounding points emulated, AdamW against a numpy
restatement, and training on a smooth regression problem."""
import numpy as np
import pytest

from oracle.mlp_oracle import MLPOracle, bf16


def test_bf16_rounding_known_values():
    x = np.array([1.0, 1.0 + 2 ** -8, 1.0 + 2 ** -7 + 2 ** -9, 3.14159265, -2.5e-3])
    r = bf16(x)
    assert r[0] == 1.0 and r[1] == 1.0  # tie to even
    assert r[2] == 1.0 + 2 ** -7  # nearest (ulp at 1 is 2^-7)
    assert abs(r[3] - 3.140625) < 1e-12
    assert abs(r[4] / -2.5e-3 - 1) < 2 ** -8


def test_oracle_gradient_matches_finite_differences():
    rng = np.random.default_rng(0)
    o = MLPOracle(n_in=13, n_hidden=16, n_hidden_layers=2, n_out=8)
    theta = rng.normal(0, 0.3, o.nparam)
    x = rng.normal(size=(5, 13))
    t = rng.normal(size=(5, 8))
    _, g = o.loss_grad(theta, x, t)
    idx = rng.choice(o.nparam, 60, replace=False)
    h = 1e-6
    for i in idx:
        tp, tm = theta.copy(), theta.copy()
        tp[i] += h
        tm[i] -= h
        fd = (o.loss_grad(tp, x, t)[0] - o.loss_grad(tm, x, t)[0]) / (2 * h)
        assert abs(fd - g[i]) <= 1e-7 + 1e-6 * abs(g[i]), (i, fd, g[i])


def _rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-30)


@pytest.mark.gpu
@pytest.mark.parametrize("gemm", ["tcgen05", "mma"])
@pytest.mark.parametrize("shape", [(30, 32, 2, 16, 70), (258, 512, 3, 128, 64),
                                   (258, 512, 3, 128, 1029)])
def test_gpu_forward_and_gradients_against_oracle(gpu_lib, monkeypatch, shape, gemm):
    """Both GEMM kernels: tcgen05 (the default) and the warp-level mma.sync
    one (COSENU_MLP_GEMM=mma).  Widths below one 64-column tile, K below one
    64-deep stage, and 1029 rows (nine 128-row tiles, the last ragged)."""
    from cosenu_b200.surrogate import MLP
    monkeypatch.setenv("COSENU_MLP_GEMM", gemm)
    n_in, nh, nl, nout, rows = shape
    rng = np.random.default_rng(1)
    net = MLP(n_in, nh, nl, nout, seed=3)
    o = MLPOracle(n_in, nh, nl, nout)
    theta = net.params().astype(np.float64)
    assert theta.size == o.nparam
    x = rng.uniform(0, 1.5, (rows, n_in)).astype(np.float32)
    t = rng.uniform(0, 1, (rows, nout)).astype(np.float32)
    y = net.forward(x)
    y_ref = o.forward(theta, x.astype(np.float64), emulate_bf16=True)[0]
    assert _rel(y, y_ref) <= 1e-3
    loss, g = net.loss_grad(x, t)
    loss_ref, g_ref = o.loss_grad(theta, x.astype(np.float64), t.astype(np.float64),
                                  emulate_bf16=True)
    assert abs(loss - loss_ref) <= 1e-3 * loss_ref
    for (ow, ob), di, do in zip(o.offsets, o.din, o.dout):
        assert _rel(g[ow:ow + di * do], g_ref[ow:ow + di * do]) <= 5e-3
        assert _rel(g[ob:ob + do], g_ref[ob:ob + do]) <= 5e-3
    # and close to the exact FP64 gradient (BF16 rounding is the only difference)
    _, g_exact = o.loss_grad(theta, x.astype(np.float64), t.astype(np.float64))
    assert _rel(g, g_exact) <= 5e-2
    net.close()


@pytest.mark.gpu
def test_gpu_adamw_step_against_numpy(gpu_lib):
    from cosenu_b200.surrogate import MLP
    rng = np.random.default_rng(2)
    net = MLP(20, 32, 2, 8, seed=5)
    o = MLPOracle(20, 32, 2, 8)
    x = rng.uniform(0, 1, (64, 20)).astype(np.float32)
    t = rng.uniform(0, 1, (64, 8)).astype(np.float32)
    w0 = net.params().astype(np.float64)
    _, g = net.loss_grad(x, t)
    lr, wd, b1, b2, eps = 1e-3, 1e-2, 0.9, 0.999, 1e-8
    net.fit(x, t, epochs=1, batch=64, lr=lr, weight_decay=wd, seed=0)
    w1 = net.params().astype(np.float64)
    m = (1 - b1) * g
    v = (1 - b2) * g.astype(np.float64) ** 2
    upd = (m / (1 - b1)) / (np.sqrt(v / (1 - b2)) + eps)
    decay = np.zeros_like(w0)
    for (ow, ob), di, do in zip(o.offsets, o.din, o.dout):
        decay[ow:ow + di * do] = wd  # weights only, not biases
    want = w0 - lr * (upd + decay * w0)
    assert np.abs(w1 - want).max() <= 1e-6
    net.close()


@pytest.mark.gpu
def test_gpu_training_fits_smooth_map(gpu_lib):
    from cosenu_b200.surrogate import MLP
    rng = np.random.default_rng(4)
    A = rng.normal(size=(24, 16)) / 4
    x = rng.uniform(-1, 1, (1024, 24)).astype(np.float32)
    t = (0.5 + 0.4 * np.sin(x @ A)).astype(np.float32)
    net = MLP(24, 128, 3, 16, seed=9)
    y0 = net.forward(x)
    base = float(np.mean((y0 - t) ** 2))
    losses = net.fit(x, t, epochs=60, batch=128, lr=2e-3, weight_decay=1e-4, seed=1)
    final = float(np.mean((net.forward(x) - t) ** 2))
    assert losses[-1] < losses[0]
    assert final < base / 20, (base, final)
    net.close()


@pytest.mark.gpu
@pytest.mark.parametrize("rows", [1, 127, 128, 129, 2053])
def test_gpu_tcgen05_gemm_matches_mma_sync_kernel(gpu_lib, monkeypatch, rows):
    """The same network evaluated with both GEMM kernels: forward outputs and
    the gradient (forward, dW = dZ^T X with both operands transposed, dX =
    dZ W with W transposed) agree to FP32 summation order and the odd BF16
    rounding flip of an activation."""
    from cosenu_b200.surrogate import MLP
    rng = np.random.default_rng(rows)
    x = rng.uniform(0, 1.5, (rows, 258)).astype(np.float32)
    t = rng.uniform(0, 1, (rows, 128)).astype(np.float32)
    out = {}
    for gemm in ("tcgen05", "mma"):
        monkeypatch.setenv("COSENU_MLP_GEMM", gemm)
        net = MLP(258, 512, 3, 128, seed=11)
        out[gemm] = (net.forward(x), net.loss_grad(x, t))
        net.close()
    (ya, (la, ga)), (yb, (lb, gb)) = out["tcgen05"], out["mma"]
    assert _rel(ya, yb) <= 2e-3
    assert abs(la - lb) <= 2e-3 * lb
    assert _rel(ga, gb) <= 5e-3

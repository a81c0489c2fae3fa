"""The fp64 oracle's training gradients (orc_step_gradients: libopenntc.cpp:651-709 in exact
arithmetic), which pin the GPU gradients, checked independently:

* central finite differences (eps 1e-3) of the oracle's own fp64 loss on 128 random g0
  latents, 128 random g1 latents and 128 random decoder weights;
* torch fp64 autograd of the same MLP on the oracle's features for dL/dW0, dL/dW1, dL/dWout.

The loss is a mean of squared residuals through hardgelu, whose derivative jumps at -1.5 and
1.5; a perturbation can move a pre-activation across a knee, so a few finite-difference
entries may miss by the jump's share, and the check allows 2 % such entries."""
import numpy as np
import pytest

F = 84  # Bpp_0_5: 4*12 + 20 + 13 rounded up to 4
C0, C1, CH = 12, 20, 9
NW = 64 * F + 64 * 64 + 16 * 64
MIP, D0, D1, TILE = 64, 16, 8, 32


def problem(seed):
    rng = np.random.default_rng(seed)
    g0 = rng.uniform(-0.6, 0.6, (D0, D0 * C0)).astype(np.float32)
    g1 = rng.uniform(-0.6, 0.6, (D1, D1 * C1)).astype(np.float32)
    W = np.zeros(NW, np.float32)
    W[:64 * F] = rng.uniform(-1, 1, 64 * F) / np.sqrt(F)
    W[64 * F:64 * F + 4096] = rng.uniform(-1, 1, 4096) / 8.0 * 2.0
    W[64 * F + 4096:] = rng.uniform(-1, 1, 16 * 64) / 8.0 * 2.0
    target = rng.integers(0, 256, (MIP, MIP * CH)).astype(np.uint8)
    return g0, g1, W, target


def build(oracle, g0, g1, W, target):
    m = oracle.model(C0, C1, F, CH, g0, g1, W, target, MIP, 2.0 / 16, 2.0 / 16)
    # the model must point at these arrays (so in-place perturbations reach it)
    assert all(a is b for a, b in zip(oracle._keep, (g0, g1, W, target)))
    return m


def loss_of(oracle, m, s):
    return oracle.step_gradients(m, s, threads=8, latent_grads=False)[0]


@pytest.mark.parametrize("seed", [1, 2])
def test_gradients_match_central_finite_differences(oracle, seed):
    g0, g1, W, target = problem(seed)
    m = build(oracle, g0, g1, W, target)
    s = oracle.step(TILE, [(7, 19)], 0, 0, 0.25)
    _, dW, dG0, dG1 = oracle.step_gradients(m, s, threads=8)
    rng = np.random.default_rng(100 + seed)
    eps = 1e-3
    for arr, grad in ((g0.reshape(-1), dG0), (g1.reshape(-1), dG1), (W, dW)):
        touched = np.flatnonzero(grad != 0)
        assert len(touched) >= 128
        idx = rng.choice(touched, 128, replace=False)
        fd = np.zeros(len(idx))
        for j, i in enumerate(idx):
            p = arr[i]
            arr[i] = p + np.float32(eps)
            hi, up = loss_of(oracle, m, s), float(arr[i])
            arr[i] = p - np.float32(eps)
            lo, dn = loss_of(oracle, m, s), float(arr[i])
            arr[i] = p
            fd[j] = (hi - lo) / (up - dn)  # the perturbation actually applied in fp32
        g = grad[idx]
        scale = np.abs(grad).max()
        # measured: worst 2.4e-6 x scale (g1 latents), median <= 2e-7 x scale
        ok = np.abs(fd - g) <= 2e-5 * scale + 1e-3 * np.abs(g)
        assert ok.mean() >= 0.98, (ok.mean(), np.abs(fd - g).max() / scale)
        assert np.median(np.abs(fd - g)) <= 1e-6 * scale


def test_decoder_gradients_match_torch_autograd(oracle):
    torch = pytest.importorskip("torch")
    g0, g1, W, target = problem(3)
    m = build(oracle, g0, g1, W, target)
    s = oracle.step(TILE, [(40, 3)], 0, 0, 0.5)
    loss, dW, _, _ = oracle.step_gradients(m, s, threads=8, latent_grads=False)
    # the oracle's own features of the step's texels (libontc's texel enumeration)
    X = np.zeros((TILE * TILE, F), np.float32)
    T = np.zeros((TILE * TILE, CH), np.float64)
    tgt = target.reshape(MIP, MIP, CH)
    for b in range(TILE * TILE):
        x, y = oracle.texel_xy(s, MIP, b)
        X[b] = oracle.features(m, s, x, y)
        T[b] = tgt[y, x] / np.float32(255.0)
    t = lambda a: torch.tensor(a, dtype=torch.float64)
    W0 = t(W[:64 * F].reshape(64, F)).requires_grad_()
    W1 = t(W[64 * F:64 * F + 4096].reshape(64, 64)).requires_grad_()
    Wo = t(W[64 * F + 4096:].reshape(16, 64)).requires_grad_()

    def hg(x):  # forward_hardgelu, ntc_kernel.cu:13-20
        return torch.where(x < -1.5, torch.zeros_like(x), torch.where(x < 1.5, x / 3 * (x + 1.5), x))

    Y = hg(hg(t(X) @ W0.T) @ W1.T) @ Wo.T
    L = ((t(T) - Y[:, :CH]) ** 2).mean()
    L.backward()
    assert abs(L.item() - loss) <= 1e-12 * loss
    got = np.concatenate([W0.grad.numpy().ravel(), W1.grad.numpy().ravel(), Wo.grad.numpy().ravel()])
    assert np.allclose(dW, got, rtol=1e-9, atol=1e-12 * np.abs(got).max())

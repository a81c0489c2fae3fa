"""The BF16 tcgen05/TMEM tile kernel against the oracle's fp64 gradients.

Tolerance: the MLP runs on bf16 operands (8-bit mantissa) with fp32 accumulation; the
feature gradient and the weight gradients are compared with a max-norm relative error
below TOL_BF16, the loss within 1 %."""
import numpy as np
import pytest

import openntc_b200 as ont
from openntc_b200 import _abi
from tests import helpers as H

pytestmark = pytest.mark.gpu

TOL_BF16 = 3e-2


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def _check(oracle, ctx, profile, step, tol=TOL_BF16, loss_tol=1e-2):
    loss = H.gradients(ctx, step)
    sh = H.shape(ctx)
    m, level = H.oracle_model(oracle, ctx, profile, step.lod)
    mip = sh["mip_dim"][step.lod]
    ost = oracle.step(min(mip, 256), [(step.ox[i], step.oy[i]) for i in range(step.n_grids)], step.noise, step.seed,
                      step.lod / (sh["mips"] - 1))
    oloss, dW, dG0, dG1 = oracle.step_gradients(m, ost)
    assert abs(loss - oloss) <= loss_tol * oloss, (loss, oloss)
    errs = {"dG0": rel_err(H.tensor(ctx, _abi.DBG_G0_GRAD, level), dG0),
            "dG1": rel_err(H.tensor(ctx, _abi.DBG_G1_GRAD, level), dG1)}
    dWd = H.tensor(ctx, _abi.DBG_W_GRAD)
    F, Cn = sh["F"], sh["C"]
    errs["dW0"] = rel_err(dWd[:64 * F], dW[:64 * F])
    errs["dW1"] = rel_err(dWd[64 * F:64 * F + 4096], dW[64 * F:64 * F + 4096])
    errs["dWout"] = rel_err(dWd[64 * F + 4096:64 * F + 4096 + Cn * 64], dW[64 * F + 4096:64 * F + 4096 + Cn * 64])
    assert not np.any(dWd[64 * F + 4096 + Cn * 64:]), "padded Wout rows must get no gradient"
    for k, v in errs.items():
        assert v < tol, (k, v, errs)
    return errs


@pytest.mark.parametrize("profile", [0, 1, 2, 3])
def test_bf16_gradients_match_oracle(materials, oracle, profile):
    ctx = H.new_context(profile, materials(256, 4, 9), min_dim=16, grids=2, steps=20, precision=ont.Precision.BF16)
    ctx.train(2)  # leave the initial state
    sh = H.shape(ctx)
    rng = np.random.default_rng(profile)
    for lod in (0, 1, sh["mips"] - 1):
        origins = [(int(rng.integers(0, sh["mip_dim"][lod])), int(rng.integers(0, sh["mip_dim"][lod]))) for _ in range(2)]
        _check(oracle, ctx, profile, H.make_step(lod, origins, noise=1, seed=77, step=5))


def test_bf16_many_units_per_cta(materials, oracle):
    """8 tiles of 256x256 = 4096 units over <= 148 CTAs: TMEM accumulation across units."""
    profile = ont.Profile.Bpp_1_0
    ctx = H.new_context(profile, materials(512, 6, 9), min_dim=16, grids=8, steps=20, precision=ont.Precision.BF16)
    step = H.make_step(0, [(i * 61, i * 37) for i in range(8)], noise=1, seed=3, step=1)
    _check(oracle, ctx, profile, step)


def test_bf16_other_channel_counts(materials, oracle):
    for ch in (4, 6, 12):
        ctx = H.new_context(ont.Profile.Bpp_0_5, materials(128, 7, ch), min_dim=16, grids=1, steps=10,
                            precision=ont.Precision.BF16)
        _check(oracle, ctx, ont.Profile.Bpp_0_5, H.make_step(0, [(5, 9)], noise=0, seed=0, step=0))


def test_bf16_training_tracks_fp32(materials):
    manifest = materials(256, 8, 9)
    res = {}
    for prec in (ont.Precision.FP32, ont.Precision.BF16):
        ctx = H.new_context(ont.Profile.Bpp_2_25, manifest, min_dim=16, grids=1, steps=400, precision=prec)
        p = ctx.train_until_complete()
        assert p.phase == ont.TrainPhase.TrainComplete and p.result == 0
        res[prec] = ctx.eval().psnr
    print("PSNR fp32 %.3f bf16 %.3f" % (res[ont.Precision.FP32], res[ont.Precision.BF16]))
    assert abs(res[ont.Precision.FP32] - res[ont.Precision.BF16]) < 0.5

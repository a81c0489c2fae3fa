"""The BF16X3 tcgen05 tile kernel (ONTC_PRECISION_BF16X3: fp32 operands split into bf16 high and
low parts, each product formed as h.h + h.l + l.h by three bf16 MMAs with fp32 accumulation,
fp32 activations) against the oracle's fp64 gradients.

Tolerance: a split product keeps about 16 mantissa bits, against 7 for bf16 (test_gpu_bf16.py
allows 3e-2) and 10 for the tf32 products of upstream's cuBLAS GEMMs (libopenntc.cpp:374); the
gradients are held to TOL_X3 max-norm relative error and the loss to 1e-4."""
import numpy as np
import pytest

import openntc_b200 as ont
from tests import helpers as H
from tests.test_gpu_bf16 import _check

pytestmark = pytest.mark.gpu

TOL_X3 = 2e-3


@pytest.mark.parametrize("profile", [0, 1, 2, 3])
def test_bf16x3_gradients_match_oracle(materials, oracle, profile):
    ctx = H.new_context(profile, materials(256, 4, 9), min_dim=16, grids=2, steps=20, precision=ont.Precision.BF16X3)
    ctx.train(2)  # leave the initial state
    sh = H.shape(ctx)
    rng = np.random.default_rng(profile)
    worst = {}
    for lod in (0, 1, sh["mips"] - 1):
        origins = [(int(rng.integers(0, sh["mip_dim"][lod])), int(rng.integers(0, sh["mip_dim"][lod]))) for _ in range(2)]
        errs = _check(oracle, ctx, profile, H.make_step(lod, origins, noise=1, seed=77, step=5), tol=TOL_X3,
                      loss_tol=1e-4)
        worst = {k: max(v, worst.get(k, 0.0)) for k, v in errs.items()}
    print(f"profile {profile} bf16x3 worst relative errors: " + ", ".join(f"{k} {v:.1e}" for k, v in worst.items()))


def test_bf16x3_many_units_per_cta(materials, oracle):
    """8 tiles of 256x256 = 4096 units over <= 148 one-group CTAs: TMEM accumulation across units."""
    profile = ont.Profile.Bpp_1_0
    ctx = H.new_context(profile, materials(512, 6, 9), min_dim=16, grids=8, steps=20,
                        precision=ont.Precision.BF16X3)
    step = H.make_step(0, [(i * 61, i * 37) for i in range(8)], noise=1, seed=3, step=1)
    _check(oracle, ctx, profile, step, tol=TOL_X3, loss_tol=1e-4)


def test_bf16x3_tracks_fp32(materials):
    """A full short schedule: BF16X3 training ends within 0.05 dB of the exact-fp32 SIMT path."""
    manifest = materials(256, 8, 9)
    res = {}
    for prec in (ont.Precision.FP32, ont.Precision.BF16X3):
        ctx = H.new_context(ont.Profile.Bpp_2_25, manifest, min_dim=16, grids=1, steps=400, precision=prec)
        p = ctx.train_until_complete()
        assert p.phase == ont.TrainPhase.TrainComplete and p.result == 0
        res[prec] = ctx.eval().psnr
        ctx.destroy()
    print("PSNR fp32 %.3f bf16x3 %.3f" % (res[ont.Precision.FP32], res[ont.Precision.BF16X3]))
    assert abs(res[ont.Precision.FP32] - res[ont.Precision.BF16X3]) < 0.05

"""BF16 batched training against the FP32 plain path on the 4096² 9-channel Bpp_1_0 set (seed 1,
4 tiles of 256² = 262,144 samples per step, the 10,000-step schedule): the final PSNR (FP64
reduction over every mip) within 0.1 dB, at three times the training samples/s or more.

Measured on a B200: PSNR 38.212 (BF16) vs 38.279 dB (FP32), 1.24 G vs 0.092 G samples/s."""
import time

import pytest

import openntc_b200 as ont

pytestmark = pytest.mark.gpu


def run(manifest, precision):
    torch = pytest.importorskip("torch")
    ctx = ont.Context()
    assert ctx.init(ont.Profile.Bpp_1_0) == ont.Result.Success
    assert ctx.load_manifest(manifest) == ont.Result.Success
    ctx.begin_training(ont.Quality.Low, 4, steps=10000, precision=precision)
    assert ctx.train(3).result == 0  # warm-up
    torch.cuda.synchronize()
    t0 = time.perf_counter()
    p = ctx.train_until_complete()
    dt = time.perf_counter() - t0
    assert p.phase == ont.TrainPhase.TrainComplete and p.batches_complete == 10000
    psnr = ctx.eval().psnr
    ctx.destroy()
    return psnr, (10000 - 3) * 4 * 256 * 256 / dt


def test_bf16_matches_fp32_plain_at_three_times_the_speed(materials):
    manifest = materials(4096, 1, 9)
    bf16, bf16_rate = run(manifest, ont.Precision.BF16)
    fp32, fp32_rate = run(manifest, ont.Precision.FP32)
    print(f"4096^2 Bpp_1_0, 10,000 steps: PSNR BF16 {bf16:.3f} dB, FP32 {fp32:.3f} dB; "
          f"{bf16_rate / 1e9:.3f} vs {fp32_rate / 1e9:.3f} G samples/s ({bf16_rate / fp32_rate:.1f}x)")
    assert abs(bf16 - fp32) <= 0.1
    assert bf16_rate >= 3.0 * fp32_rate

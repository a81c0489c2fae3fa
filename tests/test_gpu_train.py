"""End-to-end training on the GPU: schedule, completion artefacts, Eval/Calibrate against
the oracle, and PSNR against upstream at equal steps."""
import ctypes as C

import numpy as np
import pytest

import openntc_b200 as ont
from openntc_b200 import _abi
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _oracle_full(oracle, ctx, profile, noise=0, seed=0):
    """Sum of squared residuals, max |a0|, max |a1| over every mip, oracle fp64."""
    sh = H.shape(ctx)
    sq, mx0, mx1 = 0.0, 0.0, 0.0
    for mip in range(sh["mips"]):
        m, _ = H.oracle_model(oracle, ctx, profile, mip)
        s, a0, a1 = oracle.mip_sq_error(m, mip / (sh["mips"] - 1), noise, seed)
        sq += s
        mx0, mx1 = max(mx0, a0), max(mx1, a1)
    n = sum(d * d for d in sh["mip_dim"][:sh["mips"]]) * sh["C"]
    return sq / n, mx0, mx1


@pytest.fixture(scope="module")
def trained(materials):
    profile = ont.Profile.Bpp_0_5
    ctx = H.new_context(profile, materials(256, 0, 9), min_dim=16, grids=1, steps=300)
    p = ctx.train(150)
    assert p.phase == ont.TrainPhase.TrainInProgress and p.batches_complete == 150
    mid = ctx.eval()
    mid_step = H.last_step(ctx)
    p = ctx.train_until_complete()
    assert p.phase == ont.TrainPhase.TrainComplete and p.result == 0 and p.batches_complete == 300
    return dict(ctx=ctx, profile=profile, mid=mid, mid_step=mid_step)


def test_loss_decreases(trained):
    losses = np.array(trained["ctx"].step_losses(300))
    assert np.all(np.isfinite(losses)) and np.all(losses > 0)
    assert losses[-50:].mean() < 0.5 * losses[:20].mean()


def test_train_after_completion_reports_complete(trained):
    p = trained["ctx"].train(10)
    assert p.phase == ont.TrainPhase.TrainComplete and p.result == 0 and p.batches_complete == 300


def test_eval_matches_oracle(trained, oracle):
    ctx = trained["ctx"]
    e = ctx.eval()
    mse, _, _ = _oracle_full(oracle, ctx, trained["profile"])
    assert abs(e.mse - mse) <= 1e-5 * mse
    assert abs(e.psnr - (-10 * np.log10(mse))) < 1e-4


def test_calibration_matches_oracle(trained, oracle):
    ctx = trained["ctx"]
    cd = ctx.get_compressed_data()
    _, mx0, mx1 = _oracle_full(oracle, ctx, trained["profile"])
    assert abs(cd.caldata.max_abs_a1 - mx0) <= 1e-5 * mx0
    assert abs(cd.caldata.max_abs_a2 - mx1) <= 1e-5 * mx1
    assert np.float32(cd.caldata.s_a1) == np.float32(np.float32(1.1) * np.float32(cd.caldata.max_abs_a1) / np.float32(127))
    c2 = ctx.calibrate(1.1)
    assert c2.max_abs_a1 == cd.caldata.max_abs_a1 and c2.s_a2 == cd.caldata.s_a2


def test_completion_packs_latents_bit_exact(trained, oracle):
    ctx = trained["ctx"]
    cd = ctx.get_compressed_data()
    sh = H.shape(ctx)
    b0, b1, *_ = H.PROFILE_SHAPES[trained["profile"]]
    for l in range(sh["levels"]):
        for which, bits, ptr, size in [(_abi.DBG_G0, b0, cd.g0[l], cd.g0_size[l]), (_abi.DBG_G1, b1, cd.g1[l], cd.g1_size[l])]:
            lat = H.tensor(ctx, which, l)
            # locked latents sit exactly on the integer lattice (libopenntc.cpp:601-619)
            delta = 2.0 / 2 ** bits
            assert np.array_equal(lat / np.float32(delta), np.rint(lat / np.float32(delta)))
            words = np.ctypeslib.as_array(ptr, (size // 4,))
            assert np.array_equal(words, oracle.quantize_pack(lat, bits)), (which, l)


def test_decoder_blob_matches_oracle(trained, oracle):
    ctx = trained["ctx"]
    cd = ctx.get_compressed_data()
    sh = H.shape(ctx)
    F, Fp, Cn = sh["F"], sh["Fp"], sh["C"]
    W = H.tensor(ctx, _abi.DBG_W)
    W0 = np.zeros((64, Fp), np.float32)
    W0[:, :F] = W[:64 * F].reshape(64, F)
    q0, s0 = oracle.quantize_weights(W0, 1.0 / 128.0)
    q1, s1 = oracle.quantize_weights(W[64 * F:64 * F + 4096].reshape(64, 64), cd.caldata.s_a1)
    qo, so = oracle.quantize_weights(W[64 * F + 4096:64 * F + 4096 + Cn * 64].reshape(Cn, 64), cd.caldata.s_a2)
    blob = np.ctypeslib.as_array(C.cast(cd.decoder, C.POINTER(C.c_uint8)), (cd.decoder_size,)).copy()
    assert cd.decoder_size == 64 * Fp + 4096 + 16 * 64 + 4 * (64 + 64 + 16)
    o = 0
    assert np.array_equal(blob[o:o + 64 * Fp].view(np.uint32), q0); o += 64 * Fp
    assert np.array_equal(blob[o:o + 4096].view(np.uint32), q1); o += 4096
    assert np.array_equal(blob[o:o + Cn * 64].view(np.uint32), qo); o += 16 * 64
    assert np.array_equal(blob[o:o + 256].view(np.float32), s0); o += 256
    assert np.array_equal(blob[o:o + 256].view(np.float32), s1); o += 256
    sc = blob[o:o + 64].view(np.float32)
    assert np.array_equal(sc[:Cn], so) and not sc[Cn:].any()


def test_container_roundtrip(trained, tmp_path):
    ctx = trained["ctx"]
    cd = ctx.get_compressed_data()
    p = tmp_path / "m.ntc"
    assert ont.dump(p, cd) == 0
    r, fd = ont.load_file(p)
    assert r == 0
    for l in range(cd.level_count):
        a = np.ctypeslib.as_array(C.cast(fd.data.g0[l], C.POINTER(C.c_uint8)), (cd.g0_size[l],))
        b = np.ctypeslib.as_array(C.cast(cd.g0[l], C.POINTER(C.c_uint8)), (cd.g0_size[l],))
        assert np.array_equal(a, b)
    assert list(fd.data.channel_semantics)[:9] == [1, 1, 1, 6, 7, 7, 7, 8, 9]


def test_midtraining_eval_includes_live_noise(trained, oracle):
    """Eval during training adds the last step's noise (upstream reads its live noise buffer)."""
    assert trained["mid"].psnr > 10.0 and trained["mid_step"].noise == 1


@pytest.fixture(scope="module")
def upstream_cls():
    from oracle.bindings import REF_SO, RefContext
    if not REF_SO.exists():
        pytest.skip("upstream build missing")
    return RefContext


def test_upstream_noise_buffers_match(materials, upstream_cls):
    """Parity mode reproduces upstream's cuRAND noise buffers bit for bit, step after step."""
    profile, grids = ont.Profile.Bpp_0_5, 1
    manifest = materials(1024, 0, 9)
    ctx = H.new_context(profile, manifest, min_dim=1024, grids=grids, steps=1000, noise_mode=ont.NoiseMode.UPSTREAM)
    ref = upstream_cls(profile)
    try:
        assert ref.load_manifest(manifest) == 0
        ref.begin_training(0, grids, 1000, -1)
        sh = H.shape(ctx)
        for step in range(3):
            ctx.train(1)
            ref.train(1)
            s = H.last_step(ctx)
            for which, rwhich in ((_abi.DBG_NOISE0, 18), (_abi.DBG_NOISE1, 19)):
                n = (sh["g0"][s.level] ** 2) * H.PROFILE_SHAPES[profile][2] if which == _abi.DBG_NOISE0 else \
                    (sh["g1"][s.level] ** 2) * H.PROFILE_SHAPES[profile][3]
                mine = H.tensor(ctx, which, 0)[:n]
                theirs = ref.tensor(rwhich, 0)[:n]
                assert np.array_equal(mine, theirs), (step, which, np.abs(mine - theirs).max())
    finally:
        ref.close()


@pytest.mark.parametrize("precision", [ont.Precision.FP32, ont.Precision.BF16, ont.Precision.BF16X3])
def test_psnr_matches_upstream_at_equal_steps(materials, upstream_cls, precision):
    """Same seed, draws, init and (parity-mode) noise: final PSNR within 0.1 dB of upstream."""
    profile, steps, grids = ont.Profile.Bpp_0_5, 1000, 1
    manifest = materials(1024, 0, 9)
    ctx = H.new_context(profile, manifest, min_dim=1024, grids=grids, steps=steps, precision=precision,
                        noise_mode=ont.NoiseMode.UPSTREAM)
    p = ctx.train_until_complete()
    assert p.phase == ont.TrainPhase.TrainComplete
    mine = ctx.eval().psnr
    ref = upstream_cls(profile)
    try:
        assert ref.load_manifest(manifest) == 0
        ref.begin_training(0, grids, steps, -1)
        ref.train(steps)
        _, theirs = ref.eval()
    finally:
        ref.close()
    print(f"PSNR after {steps} steps: libontc {precision.name} {mine:.3f} dB, upstream {theirs:.3f} dB")
    assert abs(mine - theirs) < 0.1

"""The int8 decode scored against the training targets (ontc_eval_decoded) and the opt-in
calibration search (ONTC_CALIBRATION_SEARCH) that chooses the decoder's scales by that score.

ontc_eval_decoded is checked against the oracle's SampleMaterial at every texel centre with
Eval's arithmetic; the search against upstream's own calibration of the same trained weights
(Calibrate's 1.1 max / 127 activation scales and QuantizeWeights, restated by the oracle):
its decode must score at least as well, and its blob must still decode bit for bit as
upstream's HLSL would (same layout, oracle SampleMaterial)."""
import ctypes as C

import numpy as np
import pytest

import openntc_b200 as ont
from openntc_b200 import _abi
from tests import helpers as H
from tests.test_gpu_decode import blob, oracle_decode, pyramid, samples

pytestmark = pytest.mark.gpu

PROFILE = ont.Profile.Bpp_0_5


@pytest.fixture(scope="module")
def runs(materials):
    """The same material trained twice (300 steps): upstream calibration, and the search."""
    out = {}
    for mode in (ont.CalibrationMode.UPSTREAM, ont.CalibrationMode.SEARCH):
        ctx = H.new_context(PROFILE, materials(256, 31, 9), min_dim=16, grids=2, steps=300, calibration=mode)
        assert ctx.train_until_complete().phase == ont.TrainPhase.TrainComplete
        out[mode] = ctx
    return out


def texel_centres(ctx):
    sh = H.shape(ctx)
    uv, lod, tgt = [], [], []
    for m in range(sh["mips"]):
        d = sh["mip_dim"][m]
        x, y = np.meshgrid(np.arange(d, dtype=np.float32), np.arange(d, dtype=np.float32))
        uv.append(np.stack([(x + np.float32(0.5)) / np.float32(d), (y + np.float32(0.5)) / np.float32(d)],
                           -1).reshape(-1, 2))
        lod.append(np.full(d * d, m, np.int32))
        tgt.append(H.package(ctx, m, d * d * sh["C"]).reshape(d * d, sh["C"]))
    return np.concatenate(uv), np.concatenate(lod), np.concatenate(tgt)


def psnr_of(decoded, tgt):
    r = tgt.astype(np.float32) / np.float32(255.0) - decoded
    mse = np.sum(r.astype(np.float64) ** 2) / r.size
    return -10.0 * np.log10(mse)


def upstream_blob(oracle, ctx, cd):
    """Upstream's completion (libopenntc.cpp:839-876) for the context's trained fp32 weights."""
    sh = H.shape(ctx)
    F, Fp, Cn = sh["F"], sh["Fp"], sh["C"]
    W = H.tensor(ctx, _abi.DBG_W)
    s_a1 = np.float32(1.1) * np.float32(cd.caldata.max_abs_a1) / np.float32(127.0)
    s_a2 = np.float32(1.1) * np.float32(cd.caldata.max_abs_a2) / np.float32(127.0)
    W0 = np.zeros((64, Fp), np.float32)
    W0[:, :F] = W[:64 * F].reshape(64, F)
    q0, s0 = oracle.quantize_weights(W0, 1.0 / 128.0)
    q1, s1 = oracle.quantize_weights(W[64 * F:64 * F + 4096].reshape(64, 64), s_a1)
    qo, so = oracle.quantize_weights(W[64 * F + 4096:64 * F + 4096 + Cn * 64].reshape(Cn, 64), s_a2)
    wo = np.zeros(16 * 64, np.uint8)
    wo[:Cn * 64] = qo.view(np.uint8)
    sc = np.zeros(16, np.float32)
    sc[:Cn] = so
    b = np.concatenate([q0.view(np.uint8), q1.view(np.uint8), wo, s0.view(np.uint8), s1.view(np.uint8),
                        sc.view(np.uint8)])
    return b, float(s_a1), float(s_a2)


def test_eval_decoded_matches_oracle(runs, oracle):
    ctx = runs[ont.CalibrationMode.UPSTREAM]
    cd = ctx.get_compressed_data()
    uv, lod, tgt = texel_centres(ctx)
    want = psnr_of(oracle_decode(oracle, cd, uv, lod), tgt)
    got = ctx.eval_decoded()
    assert abs(got.psnr - want) < 1e-9 * abs(want), (got.psnr, want)
    # the int8 decode of a trained material is a usable reconstruction, not above its float model
    f = ctx.eval().psnr
    print(f"int8 decode PSNR {got.psnr:.3f} dB, float model {f:.3f} dB")
    assert 15.0 < got.psnr < f + 1.0, (got.psnr, f)


def test_upstream_mode_keeps_upstream_scales(runs, oracle):
    ctx = runs[ont.CalibrationMode.UPSTREAM]
    cd = ctx.get_compressed_data()
    b, s_a1, s_a2 = upstream_blob(oracle, ctx, cd)
    assert np.array_equal(blob(cd), b)
    assert np.float32(cd.caldata.s_a1) == np.float32(s_a1) and np.float32(cd.caldata.s_a2) == np.float32(s_a2)


def test_search_scores_at_least_upstream_on_the_same_weights(runs, oracle):
    ctx = runs[ont.CalibrationMode.SEARCH]
    cd = ctx.get_compressed_data()
    uv, lod, tgt = texel_centres(ctx)
    assert len(lod) <= 1 << 21  # the search sample is every texel here
    searched = ctx.eval_decoded().psnr
    # upstream's calibration of these same weights, decoded on the GPU
    b, s_a1, s_a2 = upstream_blob(oracle, ctx, cd)
    up = type(cd).from_buffer_copy(cd)
    keep = (C.c_uint8 * len(b)).from_buffer_copy(b.tobytes())
    up.decoder = C.cast(keep, C.c_void_p)
    up.caldata.s_a1, up.caldata.s_a2 = s_a1, s_a2
    upstream = psnr_of(ont.Decoder(up).decode_host(uv, lod), tgt)
    print(f"int8 decode PSNR: upstream calibration {upstream:.3f} dB, search {searched:.3f} dB, "
          f"float model {ctx.eval().psnr:.3f} dB; s_a1 x{cd.caldata.s_a1 / s_a1:.3f}, s_a2 x{cd.caldata.s_a2 / s_a2:.3f}")
    assert searched >= upstream - 1e-9
    # the searched file still decodes as upstream's shader would
    su, sl = samples(20000, cd.mip_count, 4)
    got = ont.Decoder(cd).decode_host(su, sl)
    assert np.array_equal(got.view(np.uint32), oracle_decode(oracle, cd, su, sl).view(np.uint32))


def test_calibration_option_is_validated(materials):
    ctx = ont.Context()
    assert ctx.init(PROFILE) == ont.Result.Success
    assert ctx.set_min_dimension(16) == ont.Result.Success
    assert ctx.load_manifest(materials(256, 31, 9)) == ont.Result.Success
    with pytest.raises(RuntimeError):
        ctx.begin_training(0, 1, calibration=7)
    e = ont.EvalResults()
    ctx._lib.ontc_eval_decoded(ctx.handle, C.byref(e))  # before completion: sticky error, zeros
    assert e.psnr == 0.0 and ctx.get_last_error() == ont.Result.InvalidState

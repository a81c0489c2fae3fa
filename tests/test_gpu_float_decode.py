"""Float-model decoders (ontc_decoder_create_float): the trained fp32 decoder weights evaluated on
the dequantised latent codes in FP32, BF16 and FP8 (e4m3, per-layer scales), against the FP64
float decode of the oracle (the same features and MLP in double, saturated), per channel."""
import ctypes as C

import numpy as np
import pytest

import openntc_b200 as ont
from openntc_b200 import _abi
from tests import helpers as H
from tests.test_gpu_decode import pyramid, samples

pytestmark = pytest.mark.gpu

# mode: (max abs error, mean abs error) bounds over every channel.  Measured on 20,037 samples of
# two 300-step materials: FP32 < 5e-6; BF16 max 3.4e-3, mean 3.4e-4; FP8 max 0.054, mean 6.8e-3.
MODES = {"fp32": (_abi.DECODE_FP32, 2e-5, 2e-6), "bf16": (_abi.DECODE_BF16, 1e-2, 1e-3),
         "fp8": (_abi.DECODE_FP8, 0.1, 0.015)}
PROFILES = [ont.Profile.Bpp_2_25, ont.Profile.Bpp_0_2]


@pytest.fixture(scope="module")
def trained(materials):
    out = {}
    for p, ch in ((ont.Profile.Bpp_2_25, 9), (ont.Profile.Bpp_0_2, 4)):
        ctx = H.new_context(p, materials(256, 41, ch), min_dim=16, grids=2, steps=300, precision=ont.Precision.BF16)
        assert ctx.train_until_complete().phase == ont.TrainPhase.TrainComplete
        out[p] = ctx
    return out


def fp64_decode(oracle, ctx, cd, uv, lod):
    k = ont.fill_constants(cd)
    return oracle.decode_float(cd.profile, pyramid(cd, 0), pyramid(cd, 1), bytes(k), H.tensor(ctx, _abi.DBG_W),
                               cd.channel_count, uv, lod)


@pytest.mark.parametrize("profile", PROFILES)
@pytest.mark.parametrize("mode", sorted(MODES))
def test_float_decode_tracks_fp64(trained, oracle, profile, mode):
    ctx = trained[profile]
    cd = ctx.get_compressed_data()
    uv, lod = samples(20000 + 37, cd.mip_count, 7)
    code, max_tol, mean_tol = MODES[mode]
    got = ont.Decoder.from_context(ctx, code).decode_host(uv, lod)
    ref = fp64_decode(oracle, ctx, cd, uv, lod)
    err = np.abs(got.astype(np.float64) - ref)
    print(f"{ont.Profile(profile).name} {mode}: max " + " ".join(f"{v:.2e}" for v in err.max(0)) +
          " mean " + " ".join(f"{v:.2e}" for v in err.mean(0)))
    assert np.all((got >= 0) & (got <= 1))
    assert err.max() <= max_tol and err.mean(0).max() <= mean_tol, (err.max(), err.mean(0).max())


def test_float_decode_device_buffers_match_host(trained):
    torch = pytest.importorskip("torch")
    ctx = trained[ont.Profile.Bpp_2_25]
    cd = ctx.get_compressed_data()
    uv, lod = samples(50000, cd.mip_count, 9)
    for code in (_abi.DECODE_FP32, _abi.DECODE_BF16, _abi.DECODE_FP8):
        dec = ont.Decoder.from_context(ctx, code)
        host = dec.decode_host(uv, lod)
        d_uv, d_lod = torch.from_numpy(uv).cuda(), torch.from_numpy(lod).cuda()
        d_out = torch.full((len(lod), cd.channel_count), -1.0, device="cuda")
        torch.cuda.synchronize()
        assert dec.decode(d_uv.data_ptr(), d_lod.data_ptr(), len(lod), d_out.data_ptr()) == 0
        assert dec.status() == 0
        assert np.array_equal(host.view(np.uint32), d_out.cpu().numpy().view(np.uint32))


def test_float_decoder_arguments(trained, materials):
    ctx = trained[ont.Profile.Bpp_2_25]
    lib = ont.load()
    h = C.c_void_p()
    assert lib.ontc_decoder_create_float(ctx.handle, _abi.DECODE_INT8, None, C.byref(h)) == ont.Result.InvalidState
    assert lib.ontc_decoder_create_float(ctx.handle, 9, None, C.byref(h)) == ont.Result.InvalidState
    fresh = H.new_context(ont.Profile.Bpp_2_25, materials(256, 41, 9), min_dim=16, grids=2, steps=300)
    assert lib.ontc_decoder_create_float(fresh.handle, _abi.DECODE_BF16, None, C.byref(h)) == ont.Result.InvalidState
    assert not h.value
    dec = ont.Decoder.from_context(ctx, _abi.DECODE_FP8)
    assert lib.ontc_decode_material(dec.handle, 1, 1, 0, 8) == ont.Result.InvalidState
    assert dec.sample_screen(8, 1, 1, 0.0, 0, 8) == ont.Result.InvalidState

"""Batch decode (ontc_decode*) against the oracle's SampleMaterial (ntc_decode.hlsli:605-623,
DP4A path): packed latents -> int8 features -> int8 MLP -> saturate, bit for bit, for every
profile, from a freshly trained material and from the same material written to and read
back from a .ntc file."""
import ctypes as C

import numpy as np
import pytest

import openntc_b200 as ont
from openntc_b200 import _abi
from tests import helpers as H

pytestmark = pytest.mark.gpu

PROFILES = [ont.Profile.Bpp_0_2, ont.Profile.Bpp_0_5, ont.Profile.Bpp_1_0, ont.Profile.Bpp_2_25]


def pyramid(cd, which):
    """The contiguous packed pyramid (levels at their byte offsets), as upstream's decoder reads it."""
    total = cd.g0_total_size if which == 0 else cd.g1_total_size
    buf = np.zeros(total // 4, np.uint32)
    for l in range(cd.level_count):
        ptr = cd.g0[l] if which == 0 else cd.g1[l]
        size = cd.g0_size[l] if which == 0 else cd.g1_size[l]
        off = cd.g0_offset[l] if which == 0 else cd.g1_offset[l]
        buf[off // 4:(off + size) // 4] = np.ctypeslib.as_array(ptr, (size // 4,))
    return buf


def blob(cd):
    return np.ctypeslib.as_array(C.cast(cd.decoder, C.POINTER(C.c_uint8)), (cd.decoder_size,)).copy()


def samples(n, mips, seed):
    rng = np.random.default_rng(seed)
    uv = rng.random((n, 2), dtype=np.float32)
    lod = rng.integers(-2, mips + 2, n).astype(np.int32)  # out-of-range lods clamp
    # edges: the texture border, exact cell centres and texel corners
    edge = np.array([[0, 0], [0.999999, 0.999999], [0.5, 0.5], [0, 0.999999], [1e-7, 0.25], [0.125, 0.875]],
                    np.float32)
    m = min(n, len(edge))
    uv[:m] = edge[:m]
    return uv, lod


def oracle_decode(oracle, cd, uv, lod):
    k = ont.fill_constants(cd)
    return oracle.sample_material(cd.profile, pyramid(cd, 0), pyramid(cd, 1), blob(cd), bytes(k), uv, lod,
                                  cd.channel_count)


@pytest.fixture(scope="module")
def trained(materials):
    """One completed material per profile (256^2, 9 channels, 60 steps)."""
    out = {}
    for p in PROFILES:
        ctx = H.new_context(p, materials(256, 7, 9), min_dim=16, grids=2, steps=60)
        prog = ctx.train_until_complete()
        assert prog.phase == ont.TrainPhase.TrainComplete and prog.result == 0
        out[p] = ctx
    return out


@pytest.mark.parametrize("profile", PROFILES)
def test_decode_matches_oracle_bit_for_bit(trained, oracle, profile):
    ctx = trained[profile]
    cd = ctx.get_compressed_data()
    uv, lod = samples(20000 + 37, cd.mip_count, int(profile))  # not a multiple of the 128-sample tile
    dec = ont.Decoder(cd)
    got = dec.decode_host(uv, lod)
    want = oracle_decode(oracle, cd, uv, lod)
    assert got.shape == want.shape == (len(lod), cd.channel_count)
    bad = np.argwhere(got.view(np.uint32) != want.view(np.uint32))
    assert len(bad) == 0, (len(bad), bad[:5], got[tuple(bad[0])], want[tuple(bad[0])])
    assert np.all((got >= 0) & (got <= 1)) and got.std() > 0.01


def test_decode_from_loaded_file_and_small_batches(trained, oracle, tmp_path):
    ctx = trained[ont.Profile.Bpp_2_25]
    cd = ctx.get_compressed_data()
    path = tmp_path / "m.ntc"
    assert ont.dump(path, cd) == 0
    r, fd = ont.load_file(path)
    assert r == 0
    dec = ont.Decoder(fd.data)
    for n in (1, 127, 128, 129, 5000):
        uv, lod = samples(n, cd.mip_count, 100 + n)
        got = dec.decode_host(uv, lod)
        assert np.array_equal(got.view(np.uint32), oracle_decode(oracle, cd, uv, lod).view(np.uint32)), n
    assert dec.decode_host(np.zeros((0, 2), np.float32), np.zeros(0, np.int32)).shape == (0, 9)


def test_decode_through_device_buffers(trained, oracle):
    torch = pytest.importorskip("torch")
    ctx = trained[ont.Profile.Bpp_1_0]
    cd = ctx.get_compressed_data()
    uv, lod = samples(70000, cd.mip_count, 5)
    stream = torch.cuda.Stream()
    dec = ont.Decoder(cd, stream.cuda_stream)
    d_uv, d_lod = torch.from_numpy(uv).cuda(), torch.from_numpy(lod).cuda()
    d_out = torch.full((len(lod), cd.channel_count), -1.0, device="cuda")
    torch.cuda.synchronize()
    assert dec.decode(d_uv.data_ptr(), d_lod.data_ptr(), len(lod), d_out.data_ptr()) == 0
    assert dec.status() == 0
    got = d_out.cpu().numpy()
    assert np.array_equal(got.view(np.uint32), oracle_decode(oracle, cd, uv, lod).view(np.uint32))


def test_int8_decode_tracks_the_float_model(trained, oracle):
    """The shipping int8 path stays close to the fp32 master model it was quantised from."""
    profile = ont.Profile.Bpp_0_5
    ctx = trained[profile]
    cd = ctx.get_compressed_data()
    uv, lod = samples(4000, cd.mip_count, 11)
    lod = np.clip(lod, 0, cd.mip_count - 1)
    got = ont.Decoder(cd).decode_host(uv, lod)
    k = ont.fill_constants(cd)
    ref = oracle.decode_float(profile, pyramid(cd, 0), pyramid(cd, 1), bytes(k), H.tensor(ctx, _abi.DBG_W),
                              cd.channel_count, uv, lod)
    err = np.abs(got - ref)
    assert err.mean() < 0.02 and err.max() < 0.25, (err.mean(), err.max())


@pytest.mark.parametrize("s_a", [(1e-3, None), (None, 1e5), (1e-3, 1e5)])
def test_decode_extreme_activation_scales(trained, oracle, s_a):
    """Activation scales whose reciprocals lie outside [1.6e-5, 600] (a hidden layer whose
    activations nearly all saturate at -128 or at 127) take the requantisation with both clamps
    and the select form of hardgelu; trained scales take the shorter form.  Both match the
    oracle bit for bit, alone and mixed across the two hidden layers."""
    ctx = trained[ont.Profile.Bpp_1_0]
    cd = type(ctx.get_compressed_data()).from_buffer_copy(ctx.get_compressed_data())
    if s_a[0] is not None:
        cd.caldata.s_a1 = s_a[0]
    if s_a[1] is not None:
        cd.caldata.s_a2 = s_a[1]
    uv, lod = samples(9000 + 11, cd.mip_count, 23)
    got = ont.Decoder(cd).decode_host(uv, lod)
    want = oracle_decode(oracle, cd, uv, lod)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_decode_uv_outside_the_unit_square(trained, oracle):
    """Coordinates outside [0, 1): the triangle-wave features come from per-CTA tables indexed
    by texel coordinate mod 8 while |floor(u * dim)| < 2^22 (negative ones too) and from the
    float formula beyond; both match the oracle bit for bit."""
    ctx = trained[ont.Profile.Bpp_2_25]
    cd = ctx.get_compressed_data()
    rng = np.random.default_rng(31)
    n = 6000
    near = rng.uniform(-3.0, 3.0, (n, 2))
    far = rng.uniform(16384.0, 40000.0, (n, 2)) * rng.choice([-1.0, 1.0], (n, 2))
    uv = np.concatenate([near, far]).astype(np.float32)
    lod = rng.integers(0, cd.mip_count, 2 * n).astype(np.int32)
    got = ont.Decoder(cd).decode_host(uv, lod)
    want = oracle_decode(oracle, cd, uv, lod)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))


def test_decoder_rejects_mismatched_data(trained):
    cd = ctx_cd = trained[ont.Profile.Bpp_0_2].get_compressed_data()
    lib = ont.load()
    h = C.c_void_p()
    bad = type(ctx_cd).from_buffer_copy(ctx_cd)
    bad.g0_bits_per_channel = 4  # Bpp_0_2 packs g0 in 2 bits
    assert lib.ontc_decoder_create(C.byref(bad), _abi.DECODE_INT8, None, C.byref(h)) == ont.Result.InvalidFile
    assert lib.ontc_decoder_create(C.byref(cd), 7, None, C.byref(h)) == ont.Result.InvalidState
    assert not h.value


def test_host_decode_pipeline_spans_chunks(trained, oracle):
    """ontc_decode_host in chunks of 2^20 samples over three streams: 3.4 M pinned samples (four
    chunks, the buffers of the first reused by the last) equal the device-buffer decode bit for
    bit, and the oracle on every 997th sample and on the chunk edges."""
    torch = pytest.importorskip("torch")
    cd = trained[ont.Profile.Bpp_2_25].get_compressed_data()
    n = 3 * (1 << 20) + 400_003
    uv, lod = samples(n, cd.mip_count, 21)
    dec = ont.Decoder(cd)
    h_uv, h_lod = torch.from_numpy(uv).pin_memory(), torch.from_numpy(lod).pin_memory()
    h_out = torch.empty((n, cd.channel_count), dtype=torch.float32).pin_memory()
    lib = ont.load()
    assert lib.ontc_decode_host(dec.handle, h_uv.data_ptr(), h_lod.data_ptr(), n, h_out.data_ptr()) == 0
    got = h_out.numpy()
    d_out = torch.empty((n, cd.channel_count), device="cuda")
    d_uv, d_lod = h_uv.cuda(), h_lod.cuda()
    torch.cuda.synchronize()
    assert dec.decode(d_uv.data_ptr(), d_lod.data_ptr(), n, d_out.data_ptr()) == 0 and dec.status() == 0
    assert np.array_equal(got.view(np.uint32), d_out.cpu().numpy().view(np.uint32))
    edges = np.array([(1 << 20) * k + o for k in range(1, 4) for o in (-1, 0)])
    idx = np.unique(np.concatenate([np.arange(0, n, 997), edges, [n - 1]]))
    want = oracle_decode(oracle, cd, uv[idx], lod[idx])
    assert np.array_equal(got[idx].view(np.uint32), want.view(np.uint32))

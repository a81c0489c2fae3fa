"""Screen-space sampling (ontc_sample_screen) and DecodeMaterial (ontc_decode_material) against
the oracle: the NTC pixel shaders' stochastic filter (flat_ntc.hlsl:74-84; ComputeLod,
StochasticFilterLod, StochasticFilterUv, InterleavedGradientNoise at ntc_decode.hlsli:143-185)
followed by SampleMaterial and DecodeMaterial (:544-623), bit for bit.

The one allowed difference: log2 is CUDA's log2f on the GPU and the C library's log2f in the
oracle; they may differ in the last bit, so a pixel whose noise value lies within 8e-6 of the
lod's fraction (lod_ab - noise within 8e-6 of an integer) may take the neighbouring integer lod.
Such a pixel must then equal the oracle's decode at that neighbouring lod."""
import numpy as np
import pytest

import openntc_b200 as ont
from tests import helpers as H
from tests.test_gpu_decode import blob, pyramid

pytestmark = pytest.mark.gpu
torch = pytest.importorskip("torch")

TIE = 8e-6


@pytest.fixture(scope="module")
def trained(materials):
    out = {}
    for p in (ont.Profile.Bpp_0_5, ont.Profile.Bpp_2_25):
        ctx = H.new_context(p, materials(256, 9, 9), min_dim=16, grids=2, steps=60)
        assert ctx.train_until_complete().phase == ont.TrainPhase.TrainComplete
        out[p] = ctx
    return out


def flat_pane(w, h):
    """flat_ntc.hlsl vs_main's uv at the pixel centres of a w x h pane."""
    x = (np.arange(w, dtype=np.float32) + 0.5) / w * 2 - 1
    y = 1 - (np.arange(h, dtype=np.float32) + 0.5) / h * 2
    nx, ny = np.meshgrid(x, y)
    a = w / h
    sx, sy = (nx * a, ny) if a >= 1 else (nx, ny / a)
    return np.stack([sx * 0.5 + 0.5, 0.5 - sy * 0.5], -1).astype(np.float32)


def ground_plane(w, h):
    """A receding plane: footprints from under a texel to many texels, strongly anisotropic."""
    t = (np.arange(h, dtype=np.float64) + 0.5) / h
    z = 1.0 / (0.02 + 0.98 * t)[:, None]
    xs = ((np.arange(w, dtype=np.float64) + 0.5) / w - 0.5)[None, :]
    u = 0.5 + xs * z * 0.25
    v = np.broadcast_to(z * 0.02, u.shape)
    return np.stack([u, v], -1).astype(np.float32)


def tiled(w, h, repeats):
    x = (np.arange(w, dtype=np.float32) + 0.5) / w * repeats
    y = (np.arange(h, dtype=np.float32) + 0.5) / h * repeats
    u, v = np.meshgrid(x, y)
    return np.stack([u, v], -1).astype(np.float32)


IMAGES = {
    "flat_333x201": lambda: flat_pane(333, 201),
    "flat_tall_97x150": lambda: flat_pane(97, 150),
    "ground_256x190": lambda: ground_plane(256, 190),
    "tiled_64x64_x8": lambda: tiled(64, 64, 8),
    "column_1x37": lambda: ground_plane(1, 37),
    "row_50x1": lambda: tiled(50, 1, 3),
}


def oracle_screen(oracle, cd, img, noise_frame, discard):
    k = ont.fill_constants(cd)
    uv, lod, keep, lod_ab, noise = oracle.screen_filter(img, cd.dim, cd.mip_count, noise_frame, discard)
    decode = lambda l: oracle.sample_material(cd.profile, pyramid(cd, 0), pyramid(cd, 1), blob(cd), bytes(k), uv,
                                              l, cd.channel_count)
    m = lod_ab.astype(np.float64) - noise.astype(np.float64)
    tie = np.abs(m - np.round(m)) < TIE
    alt = np.where(lod == np.round(m).astype(np.int32) + 1, np.round(m), np.round(m) + 1).astype(np.int32)
    alt = np.clip(alt, 0, cd.mip_count - 1)
    return decode(lod), decode(alt), keep, tie, lod


def gpu_screen(dec, img, noise_frame, flags, words):
    h, w = img.shape[:2]
    d_uv = torch.from_numpy(np.ascontiguousarray(img)).cuda()
    d_out = torch.full((h * w, words), float("nan"), device="cuda")
    torch.cuda.synchronize()
    assert dec.sample_screen(d_uv.data_ptr(), w, h, noise_frame, flags, d_out.data_ptr()) == 0
    assert dec.status() == 0
    return d_out.cpu().numpy()


def same_bits(a, b):
    return np.all(a.view(np.uint32) == b.view(np.uint32), axis=-1)


@pytest.mark.parametrize("profile", [ont.Profile.Bpp_0_5, ont.Profile.Bpp_2_25])
@pytest.mark.parametrize("name", sorted(IMAGES))
def test_screen_sampling_matches_oracle(trained, oracle, profile, name):
    cd = trained[profile].get_compressed_data()
    dec = ont.Decoder(cd)
    img = IMAGES[name]()
    for noise_frame, discard in ((0.0, False), (3.0, True)):
        want, want_alt, keep, tie, lod = oracle_screen(oracle, cd, img, noise_frame, discard)
        flags = ont.Decoder.DISCARD_OUTSIDE if discard else 0
        got = gpu_screen(dec, img, noise_frame, flags, cd.channel_count)
        # discarded pixels stay unwritten
        assert np.all(np.isnan(got[~keep]))
        ok = same_bits(got, want) | (tie & same_bits(got, want_alt))
        bad = np.flatnonzero(keep & ~ok)
        assert len(bad) == 0, (name, noise_frame, len(bad), bad[:5], lod[bad[:5]], got[bad[0]], want[bad[0]])
        assert tie.mean() < 1e-3
        if discard and name.startswith("flat_"):
            assert 0 < keep.sum() < len(keep)  # the pane is wider (or taller) than the texture


def test_stochastic_lod_choice_spans_levels(trained, oracle):
    """The receding plane spreads lods over the mip chain and the noise picks both neighbours."""
    cd = trained[ont.Profile.Bpp_2_25].get_compressed_data()
    img = ground_plane(256, 190)
    _, lod, _, lod_ab, _ = oracle.screen_filter(img, cd.dim, cd.mip_count, 1.0)
    assert lod.min() == 0 and lod.max() >= 3
    frac = lod_ab - np.floor(lod_ab)
    mixed = (frac > 0.3) & (frac < 0.7)
    assert np.any(lod[mixed] == np.floor(lod_ab[mixed])) and np.any(lod[mixed] == np.floor(lod_ab[mixed]) + 1)


@pytest.mark.parametrize("semantics", [
    None,                                 # the material's own channel semantics
    [1, 1, 1, 1, 7, 7, 9, 9, 0],          # a 4th albedo channel (dropped), 2 normal, repeated roughness, None
    [2, 5, 6, 3, 4, 8, 11, 10, 10],       # every scalar field, then a 2-channel specular
])
def test_decode_material_matches_oracle(trained, oracle, semantics):
    cd = trained[ont.Profile.Bpp_0_5].get_compressed_data()
    if semantics is not None:
        cd = type(cd).from_buffer_copy(cd)
        for i, s in enumerate(semantics):
            cd.channel_semantics[i] = s
    sem = [cd.channel_semantics[i] for i in range(cd.channel_count)]
    rng = np.random.default_rng(3)
    n = 5000 + 11
    uv = rng.random((n, 2), dtype=np.float32)
    lod = rng.integers(0, cd.mip_count, n).astype(np.int32)
    dec = ont.Decoder(cd)
    d_uv, d_lod = torch.from_numpy(uv).cuda(), torch.from_numpy(lod).cuda()
    d_out = torch.full((n, 18), float("nan"), device="cuda")
    torch.cuda.synchronize()
    assert dec.decode_material(d_uv.data_ptr(), d_lod.data_ptr(), n, d_out.data_ptr()) == 0
    assert dec.status() == 0
    got = d_out.cpu().numpy()
    k = ont.fill_constants(cd)
    ch = oracle.sample_material(cd.profile, pyramid(cd, 0), pyramid(cd, 1), blob(cd), bytes(k), uv, lod,
                                cd.channel_count)
    want = oracle.decode_material(ch, sem)
    assert np.array_equal(got.view(np.uint32), want.view(np.uint32))
    # the screen sampler's material form agrees with its channel form
    img = flat_pane(120, 90)
    chans = gpu_screen(dec, img, 2.0, 0, cd.channel_count)
    mats = gpu_screen(dec, img, 2.0, ont.Decoder.MATERIAL, 18)
    assert np.array_equal(mats.view(np.uint32), oracle.decode_material(chans, sem).view(np.uint32))


def test_sampler_argument_checks(trained):
    cd = trained[ont.Profile.Bpp_0_5].get_compressed_data()
    dec = ont.Decoder(cd)
    d = torch.zeros(64, device="cuda")
    assert dec.sample_screen(d.data_ptr(), 0, 5, 0.0, 0, d.data_ptr()) == 0  # empty image: nothing to do
    assert dec.sample_screen(d.data_ptr(), -1, 5, 0.0, 0, d.data_ptr()) == ont.Result.InvalidState
    assert dec.sample_screen(d.data_ptr(), 2, 2, 0.0, 8, d.data_ptr()) == ont.Result.InvalidState  # unknown flag
    assert dec.sample_screen(d.data_ptr() + 4, 2, 2, 0.0, 0, d.data_ptr()) == ont.Result.InvalidState  # uv not 8-aligned
    assert dec.decode_material(d.data_ptr(), d.data_ptr(), 4, d.data_ptr() + 4) == ont.Result.InvalidState

"""Arithmetic claims the kernels rest on, checked on the CPU."""
import os


def test_division_by_three_is_correctly_rounded(oracle):
    """RN(x * RN(1/3)) corrected once by the exact fma remainder equals IEEE x / 3 for every
    float with |x| <= 1.5, the only inputs hardgelu divides (2 x 1,069,547,521 values)."""
    assert oracle.L.orc_check_div3(os.cpu_count() or 1) == 0


def test_stochastic_filter_semantics(oracle):
    """The restated pixel-shader filter (ntc_decode.hlsli:143-185): over a pane whose pixels
    each span 2^2.3 texels of a 1024^2 texture, the chosen lods are 2 and 3 with mean 2.3
    (StochasticFilterLod is unbiased); a 16:1 anisotropic footprint takes its lod from
    major / 8 (max_aniso); the uv jitter stays within half the major-axis footprint."""
    import numpy as np
    dim, w, h = 1024, 128, 128
    s = 2.0 ** 2.3 / dim
    x, y = np.meshgrid((np.arange(w) + 0.5) * s, (np.arange(h) + 0.5) * s)
    img = np.stack([x, y], -1).astype(np.float32)
    uv, lod, keep, lod_ab, noise = oracle.screen_filter(img, dim, 11, 0.0)
    assert keep.all() and set(np.unique(lod)) == {2, 3}
    assert abs(lod_ab.mean() - 2.3) < 1e-3 and abs(lod.mean() - 2.3) < 0.01
    assert 0 <= noise.min() and noise.max() < 1
    assert np.abs(uv - img.reshape(-1, 2)).max() <= 0.5 * s * 1.001
    img2 = np.stack([x, y * 16], -1).astype(np.float32)  # major axis 16x the minor one
    _, lod2, _, lod_ab2, _ = oracle.screen_filter(img2, dim, 11, 0.0)
    assert abs(lod_ab2.mean() - (2.3 + 4 - 3)) < 1e-3  # log2(16 * 2^2.3 / 8)
    uv3, _, keep3, _, _ = oracle.screen_filter(img * 8, dim, 11, 0.0, True)  # uv up to 8: discarded
    assert 0 < keep3.sum() < len(keep3)


def test_box_index_quotient_by_reciprocal_is_exact():
    """The tile kernel's box loops take v / d as floor((v + 0.5) * RN(1/d)) in fp32 (div_small):
    exact for every v < 4096 and 1 <= d <= 512, which covers the staged-box item and cell indices."""
    import numpy as np
    v = np.arange(0, 4096, dtype=np.int64)
    for d in range(1, 513):
        inv = np.float32(1.0) / np.float32(d)
        q = np.floor((v.astype(np.float32) + np.float32(0.5)) * inv).astype(np.int64)
        assert np.array_equal(q, v // d), d

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


def test_hardgelu_remainder_form_equals_select_form():
    """The int8 decode's requantisation writes hardgelu as mid(max(min(x, 1.5), -1.5)) +
    (x - min(x, 1.5)) instead of x < 1.5 ? mid(max(x, -1.5)) : x.  Below 1.5 both take the same
    mid and the remainder is 0; from 1.5 up the sum is RN(mid(1.5) + RN(x - 1.5)), which must
    give back x: checked for every float in [1.5, 2^23), with mid(1.5) = 1.5 exactly.  (From
    2^23 up both forms stay at or above 2^23, which saturates.)"""
    import numpy as np
    third = np.float32(1.0) / np.float32(3.0)
    c = np.float32(1.5)
    q = c * third
    r = np.float32(np.float64(-q) * 3.0 + np.float64(c))       # fma(-q, 3, c): exact in f64 here
    q1 = np.float32(np.float64(r) * np.float64(third) + np.float64(q))
    assert q1 * (c + np.float32(1.5)) == np.float32(1.5)
    lo = np.array([1.5], np.float32).view(np.uint32)[0]
    hi = np.array([2.0 ** 23], np.float32).view(np.uint32)[0]
    step = 1 << 24
    for b in range(int(lo), int(hi), step):
        x = np.arange(b, min(b + step, int(hi)), dtype=np.uint32).view(np.float32)
        assert np.array_equal(np.float32(1.5) + (x - np.float32(1.5)), x)


def test_triangle_wave_bytes_depend_on_coordinate_mod_8():
    """The decode reads the 12 triangle-wave feature bytes from tables indexed by texel
    coordinate mod 8.  The float formula (ntc_decode.hlsli:300-330) gives the same byte for every
    integer coordinate c with |c| < 2^22, negative ones included: all of [-65536, 65536] and a
    stride through the rest of the range."""
    import numpy as np
    f32 = np.float32

    def byte(cf, p, h):
        P = f32(8 >> p)
        ph = f32(0.0) if h == 0 else f32(0.25) * P
        t = ((cf + f32(0.5)) + ph) * (f32(1.0) / P)
        pe = f32(1.0) - f32(4.0) * np.abs((t - np.floor(t)) - f32(0.5))
        return np.rint(np.clip(pe * f32(128.0), f32(-128.0), f32(127.0))).astype(np.int32)

    dense = np.arange(-65536, 65537, dtype=np.int64)
    sparse = np.arange(-(1 << 22) + 1, 1 << 22, 997, dtype=np.int64)
    c = np.concatenate([dense, sparse, [-(1 << 22) + 1, (1 << 22) - 1]])
    for p in range(3):
        for h in range(2):
            table = byte(np.arange(8, dtype=np.float32), p, h)
            assert np.array_equal(byte(c.astype(np.float32), p, h), table[c & 7]), (p, h)

"""Manifest image ingest on the host (no GPU): libontc's image loader (ontc_debug_load_image)
against upstream's own loader, stb_image's stbi_load(path, .., 4) as upstream calls it
(libopenntc.cpp:1302), exported by upstream's library built from its sources (oracle/_ref).

PNG files are written here with zlib: every colour type at every bit depth the format allows,
each of the five row filters (and a mix per row), Adam7 interlacing, odd sizes, palettes and
tRNS colour keys.  Binary PNM (the synthetic sets' format) is checked the same way, and an RGB
image must give the same pixels as PNG and as PPM.  Damaged files must fail in both loaders."""
import ctypes as C
import struct
import zlib
from pathlib import Path

import numpy as np
import pytest

import openntc_b200 as ont

ADAM7 = ((0, 0, 8, 8), (4, 0, 8, 8), (0, 4, 4, 8), (2, 0, 4, 4), (0, 2, 2, 4), (1, 0, 2, 2), (0, 1, 1, 2))
COMPS = {0: 1, 2: 3, 3: 1, 4: 2, 6: 4}


def _chunk(kind: bytes, data: bytes) -> bytes:
    return struct.pack(">I", len(data)) + kind + data + struct.pack(">I", zlib.crc32(kind + data) & 0xFFFFFFFF)


def _pack_row(samples: np.ndarray, depth: int) -> bytes:
    """One row of samples (already interleaved components) at `depth` bits, MSB first."""
    if depth == 16:
        return samples.astype(">u2").tobytes()
    if depth == 8:
        return samples.astype(np.uint8).tobytes()
    per = 8 // depth
    pad = (-len(samples)) % per
    s = np.concatenate([samples.astype(np.uint8), np.zeros(pad, np.uint8)]).reshape(-1, per)
    shifts = np.array([8 - depth * (i + 1) for i in range(per)], np.uint8)
    return (s << shifts).sum(1).astype(np.uint8).tobytes()


def _paeth(a, b, c):
    p = a + b - c
    pa, pb, pc = abs(p - a), abs(p - b), abs(p - c)
    return np.where((pa <= pb) & (pa <= pc), a, np.where(pb <= pc, b, c))


def _filter(row: bytes, prev: bytes | None, f: int, bpp: int) -> bytes:
    x = np.frombuffer(row, np.uint8).astype(np.int32)
    b = np.frombuffer(prev, np.uint8).astype(np.int32) if prev is not None else np.zeros_like(x)
    a = np.concatenate([np.zeros(bpp, np.int32), x[:-bpp]]) if len(x) > bpp else np.zeros_like(x)
    c = np.concatenate([np.zeros(bpp, np.int32), b[:-bpp]]) if len(x) > bpp else np.zeros_like(x)
    pred = {0: 0, 1: a, 2: b, 3: (a + b) >> 1, 4: _paeth(a, b, c)}[f]
    return bytes([f]) + ((x - pred) & 255).astype(np.uint8).tobytes()


def write_png(path: Path, img: np.ndarray, ctype: int, depth: int, interlace=False, filters=None,
              palette=None, trns=None, idat_split=1):
    """img: [h][w][comps] sample values (palette indices for ctype 3)."""
    h, w, comps = img.shape
    assert comps == COMPS[ctype]
    bits = comps * depth
    bpp = max(1, bits // 8)
    passes = ADAM7 if interlace else ((0, 0, 1, 1),)
    raw = b""
    row_i = 0
    for (x0, y0, dx, dy) in passes:
        sub = img[y0::dy, x0::dx]
        if sub.shape[0] == 0 or sub.shape[1] == 0:
            continue
        prev = None
        for y in range(sub.shape[0]):
            row = _pack_row(sub[y].reshape(-1), depth)
            f = (filters[row_i % len(filters)] if filters is not None else row_i % 5)
            raw += _filter(row, prev, f, bpp)
            prev = row
            row_i += 1
    z = zlib.compress(raw, 9)
    out = b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", w, h, depth, ctype, 0, 0, int(interlace)))
    if palette is not None:
        out += _chunk(b"PLTE", bytes(np.asarray(palette, np.uint8).reshape(-1)))
    if trns is not None:
        out += _chunk(b"tRNS", bytes(trns))
    step = max(1, (len(z) + idat_split - 1) // idat_split)
    for i in range(0, len(z), step):
        out += _chunk(b"IDAT", z[i:i + step])
    out += _chunk(b"IEND", b"")
    path.write_bytes(out)
    return path


@pytest.fixture(scope="module")
def stb():
    from oracle.bindings import REF_SO
    if not REF_SO.exists():
        pytest.skip(f"{REF_SO} not built")
    L = C.CDLL(str(REF_SO))
    L.stbi_load.restype = C.POINTER(C.c_uint8)
    L.stbi_load.argtypes = [C.c_char_p, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int), C.c_int]
    L.stbi_image_free.argtypes = [C.c_void_p]

    def load(path):
        w, h, c = C.c_int(), C.c_int(), C.c_int()
        p = L.stbi_load(str(path).encode(), C.byref(w), C.byref(h), C.byref(c), 4)
        if not p:
            return None
        out = np.ctypeslib.as_array(p, (h.value, w.value, 4)).copy()
        L.stbi_image_free(p)
        return out

    return load


def ours(path):
    lib = ont.load()
    w, h = C.c_int32(), C.c_int32()
    r = lib.ontc_debug_load_image(str(path).encode(), C.byref(w), C.byref(h), None)
    if r != 0:
        assert r == ont.Result.FileNotFound
        return None
    out = np.zeros((h.value, w.value, 4), np.uint8)
    assert lib.ontc_debug_load_image(str(path).encode(), C.byref(w), C.byref(h), out.ctypes.data_as(C.c_void_p)) == 0
    return out


def _cases(rng):
    sizes = [(1, 1), (7, 13), (17, 9), (33, 32), (64, 5)]
    for ctype, depths in ((0, (1, 2, 4, 8, 16)), (2, (8, 16)), (3, (1, 2, 4, 8)), (4, (8, 16)), (6, (8, 16))):
        for depth in depths:
            for (h, w) in sizes:
                for interlace in (False, True):
                    hi = (1 << depth) - 1
                    img = rng.integers(0, hi + 1, (h, w, COMPS[ctype]), dtype=np.int64)
                    if ctype == 3:
                        n = 1 << depth
                        pal = rng.integers(0, 256, (n, 3))
                        yield dict(img=img, ctype=ctype, depth=depth, interlace=interlace, palette=pal,
                                   trns=list(rng.integers(0, 256, n // 2 + 1)) if h * w > 1 else None)
                    else:
                        trns = None
                        if ctype in (0, 2) and w > 3:  # a colour key that some pixels carry
                            keypix = img[0, 1]
                            trns = b"".join(struct.pack(">H", int(v)) for v in keypix)
                        yield dict(img=img, ctype=ctype, depth=depth, interlace=interlace, trns=trns)


def test_png_matches_upstream_stb_image(tmp_path, stb):
    rng = np.random.default_rng(7)
    n = 0
    for i, case in enumerate(_cases(rng)):
        filters = [i % 5] if i % 3 else None  # one filter on every row, or all five in turn
        p = write_png(tmp_path / f"c{i}.png", case["img"], case["ctype"], case["depth"], case["interlace"],
                      filters=filters, palette=case.get("palette"), trns=case.get("trns"), idat_split=1 + i % 3)
        want = stb(p)
        assert want is not None, case
        got = ours(p)
        assert got is not None, {k: case[k] for k in ("ctype", "depth", "interlace")}
        assert np.array_equal(got, want), ({k: case[k] for k in ("ctype", "depth", "interlace")}, case["img"].shape)
        n += 1
    assert n == 150


def test_pnm_matches_upstream_stb_image(tmp_path, stb):
    rng = np.random.default_rng(8)
    for i, (h, w, c) in enumerate([(1, 1, 1), (5, 9, 3), (32, 32, 1), (31, 17, 3)]):
        img = rng.integers(0, 256, (h, w, c), dtype=np.uint8)
        head = b"P5" if c == 1 else b"P6"
        p = tmp_path / f"i{i}.pnm"
        p.write_bytes(head + b"\n# a comment\n%d %d\n255\n" % (w, h) + img.tobytes())
        assert np.array_equal(ours(p), stb(p))


def test_png_and_ppm_give_the_same_pixels(tmp_path):
    rng = np.random.default_rng(9)
    img = rng.integers(0, 256, (48, 40, 3), dtype=np.uint8)
    ppm = tmp_path / "a.ppm"
    ppm.write_bytes(b"P6\n40 48\n255\n" + img.tobytes())
    for f in range(5):
        png = write_png(tmp_path / f"a{f}.png", img.astype(np.int64), 2, 8, filters=[f])
        assert np.array_equal(ours(png), ours(ppm)), f
    expect = np.concatenate([img, np.full((48, 40, 1), 255, np.uint8)], -1)
    assert np.array_equal(ours(ppm), expect)


def test_damaged_files_fail_in_both_loaders(tmp_path, stb):
    rng = np.random.default_rng(10)
    img = rng.integers(0, 256, (16, 16, 3), dtype=np.int64)
    good = write_png(tmp_path / "good.png", img, 2, 8).read_bytes()
    sig_end = 8 + 25  # signature + IHDR chunk
    damaged = {
        "truncated_idat": good[:sig_end + 30],
        "bad_filter_byte": None,
        "no_idat": good[:sig_end] + _chunk(b"IEND", b""),
        "not_an_image": b"hello world, not an image at all",
        "empty": b"",
        "bad_colour_type": good[:8] + _chunk(b"IHDR", struct.pack(">IIBBBBB", 16, 16, 8, 5, 0, 0, 0)) + good[sig_end:],
        "bad_depth": good[:8] + _chunk(b"IHDR", struct.pack(">IIBBBBB", 16, 16, 4, 2, 0, 0, 0)) + good[sig_end:],
        "pnm_short": b"P6\n16 16\n255\n" + bytes(100),
    }
    raw = b""
    for y in range(16):
        raw += bytes([7]) + img[y].astype(np.uint8).tobytes()  # filter type 7 does not exist
    damaged["bad_filter_byte"] = (b"\x89PNG\r\n\x1a\n" + _chunk(b"IHDR", struct.pack(">IIBBBBB", 16, 16, 8, 2, 0, 0, 0))
                                  + _chunk(b"IDAT", zlib.compress(raw)) + _chunk(b"IEND", b""))
    for name, data in damaged.items():
        p = tmp_path / f"{name}.png"
        p.write_bytes(data)
        assert stb(p) is None, name
        assert ours(p) is None, name
    assert ours(tmp_path / "does_not_exist.png") is None

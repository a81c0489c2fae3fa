"""Seeded synthetic PBR material sets (stand-ins for the texture sets upstream's README
quotes, which are not distributed with the source).

A set is a directory of binary PNM images plus a manifest.json in upstream's manifest format
(README.md:19-43).  The fields:

  * height: 6-octave value noise (lacunarity 2, gain 0.5), smoothstep-interpolated lattices;
  * Albedo RGB: height through a 3-stop colour ramp plus U(-0.03, 0.03) noise, 8-bit;
  * Normal RGB: normalised height gradient packed to 8 bits;
  * Roughness: a second noise field mapped to [0.2, 0.9];
  * Metallic: a third noise field thresholded to {0, 1};
  * AO: 1 - 0.5 * cavity (positive part of height minus its local blur);
  * Specular RGB (12-channel sets only): a fourth field through a grey ramp.

Channel counts: 4 = Albedo + Roughness, 6 = Albedo + Normal, 9 = Albedo + Normal +
Roughness + Metallic + AO, 12 = the 9 plus Specular.
"""
from __future__ import annotations

import json
import os
from pathlib import Path

import numpy as np


def value_noise(dim: int, rng: np.random.Generator, octaves: int = 6, base: int = 4,
                lacunarity: float = 2.0, gain: float = 0.5) -> np.ndarray:
    """Fractal value noise in [0, 1], float32 [dim][dim], tileable."""
    out = np.zeros((dim, dim), np.float32)
    amp, freq, norm = 1.0, float(base), 0.0
    coords = (np.arange(dim, dtype=np.float32) + 0.5) / dim
    for _ in range(octaves):
        f = max(1, int(round(freq)))
        lat = rng.random((f, f), dtype=np.float32)
        p = coords * f - 0.5
        i0 = np.floor(p).astype(np.int64)
        t = p - i0
        t = t * t * (3.0 - 2.0 * t)
        a, b = i0 % f, (i0 + 1) % f
        rows = lat[a][:, a] * (1 - t)[None, :] + lat[a][:, b] * t[None, :]
        rows2 = lat[b][:, a] * (1 - t)[None, :] + lat[b][:, b] * t[None, :]
        out += amp * (rows * (1 - t)[:, None] + rows2 * t[:, None])
        norm += amp
        amp *= gain
        freq *= lacunarity
    return out / norm


def _box_blur(x: np.ndarray, r: int) -> np.ndarray:
    k = 2 * r + 1
    c = np.cumsum(np.pad(x, ((r + 1, r), (0, 0)), mode="wrap"), axis=0)
    x = (c[k:] - c[:-k]) / k
    c = np.cumsum(np.pad(x, ((0, 0), (r + 1, r)), mode="wrap"), axis=1)
    return (c[:, k:] - c[:, :-k]) / k


def _u8(x: np.ndarray) -> np.ndarray:
    return np.clip(np.rint(x * 255.0), 0, 255).astype(np.uint8)


def _write_pnm(path: Path, img: np.ndarray):
    if img.ndim == 2:
        head = b"P5\n%d %d\n255\n" % (img.shape[1], img.shape[0])
    else:
        head = b"P6\n%d %d\n255\n" % (img.shape[1], img.shape[0])
    with open(path, "wb") as f:
        f.write(head)
        f.write(np.ascontiguousarray(img).tobytes())


def make_material(out_dir: str | os.PathLike, dim: int, seed: int, channels: int = 9) -> Path:
    """Writes a material set and returns the manifest path.  Deterministic in (dim, seed)."""
    assert channels in (4, 6, 9, 12)
    out = Path(out_dir)
    out.mkdir(parents=True, exist_ok=True)
    rng = np.random.default_rng(seed)
    h = value_noise(dim, rng)
    ramp = np.array([[0.35, 0.22, 0.12], [0.62, 0.55, 0.42], [0.86, 0.84, 0.78]], np.float32)
    t = np.clip(h, 0, 1) * 2.0
    lo = np.clip(np.floor(t).astype(np.int64), 0, 1)
    fr = (t - lo)[..., None]
    albedo = ramp[lo] * (1 - fr) + ramp[lo + 1] * fr
    albedo = albedo + rng.uniform(-0.03, 0.03, size=albedo.shape).astype(np.float32)
    gy, gx = np.gradient(h * 8.0)
    n = np.stack([-gx * dim / 64.0, -gy * dim / 64.0, np.ones_like(h)], -1)
    n /= np.linalg.norm(n, axis=-1, keepdims=True)
    normal = n * 0.5 + 0.5
    rough = 0.2 + 0.7 * value_noise(dim, rng)
    metal = (value_noise(dim, rng) > 0.55).astype(np.float32)
    cavity = np.maximum(_box_blur(h, max(1, dim // 256)) - h, 0.0)
    ao = 1.0 - 0.5 * np.clip(cavity * 8.0, 0.0, 1.0)

    textures = []
    _write_pnm(out / "BaseColor.ppm", _u8(albedo))
    textures.append({"fileName": "BaseColor.ppm", "isSRGB": True, "semantics": {"Albedo": "RGB"}})
    if channels in (6, 9, 12):
        _write_pnm(out / "Normal.ppm", _u8(normal))
        textures.append({"fileName": "Normal.ppm", "semantics": {"Normal": "RGB"}})
    if channels in (4, 9, 12):
        rm = np.stack([np.zeros_like(rough), rough, metal], -1)
        _write_pnm(out / "RoughnessMetalness.ppm", _u8(rm))
        sem = {"Roughness": "G"} if channels == 4 else {"Roughness": "G", "Metallic": "B"}
        textures.append({"fileName": "RoughnessMetalness.ppm", "semantics": sem})
    if channels in (9, 12):
        _write_pnm(out / "AmbientOcclusion.pgm", _u8(ao))
        textures.append({"fileName": "AmbientOcclusion.pgm", "semantics": {"Occlusion": "R"}})
    if channels == 12:
        sp = value_noise(dim, rng)
        spec = np.stack([sp * 0.5 + 0.25, sp * 0.45 + 0.25, sp * 0.4 + 0.3], -1)
        _write_pnm(out / "Specular.ppm", _u8(spec))
        textures.append({"fileName": "Specular.ppm", "semantics": {"Specular": "RGB"}})
    # upstream resolves fileName against the working directory; absolute paths keep the
    # manifest usable from anywhere
    for t in textures:
        t["fileName"] = str((out / t["fileName"]).resolve())
    manifest = {"width": dim, "height": dim, "textures": textures}
    mpath = out / "manifest.json"
    mpath.write_text(json.dumps(manifest, indent=2))
    return mpath

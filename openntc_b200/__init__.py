"""openntc_b200 -- B200-native neural texture compression (training + decode).

Python mirror of upstream's libopenntc interface (libopenntc/libopenntc.h:168-197,
libopenntc/openntc_runtime.h:55-150) over the C ABI of the in-tree libontc.so.  All compute
runs in libontc.so's sm_100a kernels; importing this package never falls back to anything
else: if libontc.so is missing, load() raises.

    ctx = Context()
    ctx.init(Profile.Bpp_0_5)
    ctx.load_manifest("manifest.json")
    ctx.begin_training(Quality.Medium, grids_per_batch=1)
    ctx.train_until_complete()
    print(ctx.eval().psnr)
    dump("out.ntc", ctx.get_compressed_data())
"""
from __future__ import annotations

import ctypes as C
import enum
import os
from pathlib import Path

from . import _abi
from ._abi import (CompressedData, Constants, EvalResults, TextureData, TrainOptions,  # noqa: F401
                   TrainProgress, Calibration)

LIB_PATH = Path(__file__).resolve().parent / "libontc.so"
_lib = None


class Profile(enum.IntEnum):
    """openntc::Profile (openntc_runtime.h:8-16)."""
    Bpp_0_2 = 0
    Bpp_0_5 = 1
    Bpp_1_0 = 2
    Bpp_2_25 = 3


class Quality(enum.IntEnum):
    """openntc::Quality (libopenntc.h:147-155)."""
    Low = 0
    Medium = 1
    High = 2
    Ultra = 3


class Result(enum.IntEnum):
    """openntc::Result (openntc_runtime.h:18-30)."""
    Success = 0
    InvalidDimension = 1
    AllocationFailure = 2
    InvalidManifest = 3
    FileNotFound = 4
    InvalidFile = 5
    FileWriteFailure = 6
    InvalidState = 7
    CudaFailure = 8


class TrainPhase(enum.IntEnum):
    """openntc::TrainPhase (libopenntc.h:99-106)."""
    ManifestLoaded = 0
    TrainInProgress = 1
    TrainComplete = 2
    TrainError = -1


class Precision(enum.IntEnum):
    BF16 = 0
    FP32 = 1
    BF16X3 = 2


class LatentAdam(enum.IntEnum):
    DEFERRED = 0  # footprint updates + exact replay of the zero-gradient steps
    DENSE = 1     # one pass over the whole level every step


class CalibrationMode(enum.IntEnum):
    UPSTREAM = 0  # Calibrate's 1.1 max / 127 activation scales, per-row max weight scales
    SEARCH = 1    # scales chosen by the int8 decode's error on a texel sample


class NoiseMode(enum.IntEnum):
    COUNTER = 0   # counter-based surrogate, generated at the touched latents only
    UPSTREAM = 1  # upstream's cuRAND stream and level-wide buffers (trajectory parity)


def load() -> C.CDLL:
    """Loads (once) and binds the in-tree libontc.so.  Raises if it was not built."""
    global _lib
    if _lib is None:
        if not LIB_PATH.exists():
            raise RuntimeError(f"{LIB_PATH} is missing: run `python -m openntc_b200.build` first")
        _lib = _abi.bind(C.CDLL(str(LIB_PATH)))
    return _lib


class Context:
    """openntc::Context (libopenntc.h:168-197) over the C ABI."""

    def __init__(self):
        self._lib = load()
        self._h = self._lib.ontc_create()

    def __del__(self):
        self.destroy()

    def destroy(self):
        if getattr(self, "_h", None):
            self._lib.ontc_destroy(self._h)
            self._h = None

    @property
    def handle(self):
        return self._h

    def init(self, profile: int, stream: int | None = None) -> Result:
        return Result(self._lib.ontc_init(self._h, int(profile), C.c_void_p(stream or 0)))

    def set_min_dimension(self, dim: int) -> Result:
        return Result(self._lib.ontc_set_min_dimension(self._h, dim))

    def load_manifest(self, path: str | os.PathLike) -> Result:
        return Result(self._lib.ontc_load_manifest(self._h, str(path).encode()))

    def unload_manifest(self):
        self._lib.ontc_unload_manifest(self._h)

    def begin_training(self, quality: int, grids_per_batch: int = 1, steps: int | None = None,
                       lock_step: int | None = None, precision: int = Precision.BF16,
                       noise_mode: int = NoiseMode.COUNTER, latent_adam: int = LatentAdam.DEFERRED,
                       calibration: int = CalibrationMode.UPSTREAM):
        self._lib.ontc_begin_training(self._h, int(quality), int(grids_per_batch))
        o = TrainOptions()
        o.steps_override = steps or 0
        o.has_lock_step = 1 if lock_step is not None else 0
        o.lock_step = lock_step or 0
        o.precision = int(precision)
        o.noise_mode = int(noise_mode)
        o.latent_adam = int(latent_adam)
        o.calibration = int(calibration)
        r = self._lib.ontc_set_train_options(self._h, C.byref(o))
        if r != 0:
            raise RuntimeError(f"ontc_set_train_options: {Result(r).name}")

    def train(self, num_batches: int) -> TrainProgress:
        p = TrainProgress()
        self._lib.ontc_train(self._h, int(num_batches), C.byref(p))
        return p

    def train_until_complete(self) -> TrainProgress:
        p = TrainProgress()
        self._lib.ontc_train_until_complete(self._h, C.byref(p))
        return p

    def eval(self) -> EvalResults:
        r = EvalResults()
        self._lib.ontc_eval(self._h, C.byref(r))
        return r

    def eval_decoded(self) -> EvalResults:
        """PSNR of the shipping int8 decode over every texel of every mip (after completion)."""
        r = EvalResults()
        self._lib.ontc_eval_decoded(self._h, C.byref(r))
        return r

    def calibrate(self, headroom: float = 1.1) -> Calibration:
        c = Calibration()
        self._lib.ontc_calibrate(self._h, headroom, C.byref(c))
        return c

    def get_compressed_data(self) -> CompressedData:
        d = CompressedData()
        self._lib.ontc_get_compressed_data(self._h, C.byref(d))
        return d

    def get_texture_data(self) -> TextureData:
        t = TextureData()
        self._lib.ontc_get_texture_data(self._h, C.byref(t))
        return t

    def get_mip_dim(self, mip: int) -> int:
        return self._lib.ontc_get_mip_dim(self._h, mip)

    def feature_level_for_lod(self, lod: int) -> int:
        return self._lib.ontc_feature_level_for_lod(self._h, lod)

    def get_last_error(self) -> Result:
        return Result(self._lib.ontc_get_last_error(self._h))

    def step_losses(self, n: int):
        buf = (C.c_double * n)()
        r = self._lib.ontc_get_step_losses(self._h, buf, n)
        if r != 0:
            raise RuntimeError(f"ontc_get_step_losses: {Result(r).name}")
        return list(buf)

    def kernel_launches(self) -> int:
        return self._lib.ontc_kernel_launch_count(self._h)

    def texels_trained(self) -> int:
        """Texels actually trained so far (a step at a mip below 256^2 trains fewer)."""
        return self._lib.ontc_texels_trained(self._h)


class FileData:
    """openntc::FileData (openntc_runtime.h:131-150): owns a loaded container."""

    def __init__(self):
        self._lib = load()
        self._h = C.c_void_p()
        self.data = CompressedData()

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ontc_file_free(self._h)
            self._h = None


def dump(path: str | os.PathLike, data: CompressedData) -> Result:
    """openntc::Dump (openntc_runtime.cpp:179)."""
    return Result(load().ontc_dump(str(path).encode(), C.byref(data)))


def load_file(path: str | os.PathLike) -> tuple[Result, FileData]:
    """openntc::Load (openntc_runtime.cpp:307)."""
    fd = FileData()
    r = load().ontc_load(str(path).encode(), C.byref(fd._h), C.byref(fd.data))
    return Result(r), fd


def fill_constants(data: CompressedData) -> Constants:
    """openntc::FillNTCConstants (openntc_runtime.cpp:156)."""
    c = Constants()
    load().ontc_fill_constants(C.byref(data), C.byref(c))
    return c


def train_batch(contexts: list, num_batches: int) -> tuple[Result, list]:
    """Advances every context by up to num_batches steps, overlapping their GPU work
    (ontc_train_batch).  Returns the overall result and each context's TrainProgress."""
    lib = load()
    n = len(contexts)
    hs = (C.c_void_p * n)(*[c.handle for c in contexts])
    out = (TrainProgress * n)()
    r = lib.ontc_train_batch(hs, n, int(num_batches), out)
    return Result(r), list(out)


class Decoder:
    """Batch SampleMaterial (ntc_decode.hlsli:605-623) of one compressed material on the GPU."""

    DISCARD_OUTSIDE = _abi.SCREEN_DISCARD_OUTSIDE  # sample_screen flags
    MATERIAL = _abi.SCREEN_MATERIAL

    def __init__(self, data: CompressedData, stream: int | None = None):
        self._lib = load()
        h = C.c_void_p()
        r = self._lib.ontc_decoder_create(C.byref(data), _abi.DECODE_INT8, stream, C.byref(h))
        if r != 0:
            raise RuntimeError(f"ontc_decoder_create failed: {Result(r).name}")
        self._h = h.value
        self.channels = data.channel_count

    @classmethod
    def from_context(cls, ctx: "Context", mode: int, stream: int | None = None) -> "Decoder":
        """A decoder of a trained context's float model: mode _abi.DECODE_FP32 / BF16 / FP8."""
        self = cls.__new__(cls)
        self._lib = load()
        h = C.c_void_p()
        r = self._lib.ontc_decoder_create_float(ctx.handle, int(mode), stream, C.byref(h))
        if r != 0:
            raise RuntimeError(f"ontc_decoder_create_float failed: {Result(r).name}")
        self._h = h.value
        self.channels = ctx.get_compressed_data().channel_count
        return self

    def __del__(self):
        if getattr(self, "_h", None):
            self._lib.ontc_decoder_destroy(self._h)
            self._h = None

    @property
    def handle(self) -> int:
        return self._h

    def decode_host(self, uv, lod):
        """uv: float32 [n, 2], lod: int32 [n] (numpy) -> float32 [n, channels]."""
        import numpy as np
        uv = np.ascontiguousarray(uv, np.float32)
        lod = np.ascontiguousarray(lod, np.int32)
        out = np.empty((len(lod), self.channels), np.float32)
        r = self._lib.ontc_decode_host(self._h, uv.ctypes.data, lod.ctypes.data, len(lod), out.ctypes.data)
        if r != 0:
            raise RuntimeError(f"ontc_decode_host failed: {Result(r).name}")
        return out

    def decode(self, d_uv: int, d_lod: int, n: int, d_out: int) -> Result:
        """Device pointers; enqueued on the decoder's stream."""
        return Result(self._lib.ontc_decode(self._h, d_uv, d_lod, n, d_out))

    def status(self) -> Result:
        return Result(self._lib.ontc_decoder_status(self._h))

    def decode_material(self, d_uv: int, d_lod: int, n: int, d_params: int) -> Result:
        """SampleMaterial with DecodeMaterial: d_params is ontc_material_params [n] (18 words each)."""
        return Result(self._lib.ontc_decode_material(self._h, d_uv, d_lod, n, d_params))

    def sample_screen(self, d_uv: int, width: int, height: int, noise_frame: float, flags: int, d_out: int) -> Result:
        """Stochastic screen-space sampling of a [height][width][2] uv image (device pointers);
        flags: SCREEN_DISCARD_OUTSIDE | SCREEN_MATERIAL."""
        return Result(self._lib.ontc_sample_screen(self._h, d_uv, width, height, noise_frame, flags, d_out))


def semantic_from_name(name: str) -> int:
    return load().ontc_semantic_from_name(name.encode())


def semantic_to_string(sem: int) -> str:
    return load().ontc_semantic_to_string(sem).decode()


def profile_to_string(p: int) -> str:
    return load().ontc_profile_to_string(p).decode()


def profile_from_string(s: str):
    out = C.c_int32()
    ok = load().ontc_profile_from_string(s.encode(), C.byref(out))
    return out.value if ok else None


def channel_count_for_semantic(sem: int) -> int:
    return load().ontc_channel_count_for_semantic(sem)


def steps_for_quality(q: int) -> int:
    return load().ontc_steps_for_quality(q)

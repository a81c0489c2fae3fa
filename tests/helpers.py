"""Shared helpers for the tests: libontc introspection through the C ABI."""
from __future__ import annotations

import ctypes as C

import numpy as np

import openntc_b200 as ont
from openntc_b200 import _abi

PROFILE_SHAPES = {  # profile -> (b0, b1, C0, C1, scale)   libopenntc.cpp:289-328
    0: (2, 4, 8, 12, 4),
    1: (4, 4, 12, 20, 4),
    2: (2, 4, 12, 10, 2),
    3: (4, 4, 16, 12, 2),
}


def feature_dim(profile: int) -> int:
    b0, b1, C0, C1, _ = PROFILE_SHAPES[profile]
    return ((4 * C0 + C1 + 13 + 3) // 4) * 4


def shape(ctx: ont.Context) -> dict:
    o = np.zeros(33, np.int32)
    ctx._lib.ontc_debug_shape(ctx.handle, o.ctypes.data_as(C.c_void_p))
    return {"F": int(o[0]), "Fp": int(o[1]), "C": int(o[2]), "mips": int(o[3]), "levels": int(o[4]), "nW": int(o[5]),
            "g0": [int(v) for v in o[6:12]], "g1": [int(v) for v in o[12:18]],
            "mip_dim": [int(v) for v in o[18:30]], "batch_i": int(o[30]), "lock_i": int(o[31]),
            "batch_count": int(o[32])}


def tensor(ctx: ont.Context, which: int, level: int = 0) -> np.ndarray:
    n = ctx._lib.ontc_debug_tensor(ctx.handle, which, level, None, 0, 0)
    assert n > 0, (which, level, n)
    out = np.zeros(n, np.float32)
    got = ctx._lib.ontc_debug_tensor(ctx.handle, which, level, out.ctypes.data_as(C.c_void_p), n, 0)
    assert got == n
    return out


def set_tensor(ctx: ont.Context, which: int, level: int, data: np.ndarray):
    data = np.ascontiguousarray(data, np.float32)
    got = ctx._lib.ontc_debug_tensor(ctx.handle, which, level, data.ctypes.data_as(C.c_void_p), data.size, 1)
    assert got == data.size


def last_step(ctx: ont.Context) -> _abi.DebugStep:
    s = _abi.DebugStep()
    ctx._lib.ontc_debug_last_step(ctx.handle, C.byref(s))
    return s


def gradients(ctx: ont.Context, step: _abi.DebugStep):
    loss = C.c_double()
    r = ctx._lib.ontc_debug_gradients(ctx.handle, C.byref(step), C.byref(loss))
    assert r == 0, ont.Result(r).name
    return loss.value


def package(ctx: ont.Context, mip: int, size: int) -> np.ndarray:
    out = np.zeros(size, np.uint8)
    assert ctx._lib.ontc_debug_package(ctx.handle, mip, out.ctypes.data_as(C.c_void_p)) == 0
    return out


def make_step(lod, origins, noise=0, seed=0, step=0) -> _abi.DebugStep:
    s = _abi.DebugStep()
    s.lod = lod
    s.n_grids = len(origins)
    for i, (x, y) in enumerate(origins):
        s.ox[i], s.oy[i] = x, y
    s.noise, s.seed, s.step = noise, seed, step
    return s


def new_context(profile: int, manifest, min_dim: int = 16, quality: int = 0, grids: int = 1, steps=None,
                lock_step=None, precision=ont.Precision.FP32, noise_mode=ont.NoiseMode.COUNTER,
                latent_adam=ont.LatentAdam.DEFERRED, calibration=ont.CalibrationMode.UPSTREAM) -> ont.Context:
    ctx = ont.Context()
    r = ctx.init(profile)
    assert r == ont.Result.Success, r
    assert ctx.set_min_dimension(min_dim) == ont.Result.Success
    r = ctx.load_manifest(manifest)
    assert r == ont.Result.Success, r
    ctx.begin_training(quality, grids, steps=steps, lock_step=lock_step, precision=precision, noise_mode=noise_mode,
                       latent_adam=latent_adam, calibration=calibration)
    return ctx


def oracle_model(oracle, ctx: ont.Context, profile: int, lod: int, target: np.ndarray | None = None):
    """An oracle model bound to the context's current state at the level serving `lod`."""
    sh = shape(ctx)
    b0, b1, C0, C1, _ = PROFILE_SHAPES[profile]
    level = ctx.feature_level_for_lod(lod)
    g0 = tensor(ctx, _abi.DBG_G0, level)
    g1 = tensor(ctx, _abi.DBG_G1, level)
    W = tensor(ctx, _abi.DBG_W)
    mip = sh["mip_dim"][lod]
    if target is None:
        target = package(ctx, lod, mip * mip * sh["C"])
    m = oracle.model(C0, C1, sh["F"], sh["C"], g0.reshape(sh["g0"][level], -1), g1.reshape(sh["g1"][level], -1), W,
                     target, mip, 2.0 / 2 ** b0, 2.0 / 2 ** b1)
    return m, level

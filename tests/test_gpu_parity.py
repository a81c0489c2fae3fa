"""GPU parity of libontc's kernels against the CPU oracle and against upstream compiled
from its own sources (oracle/_ref).  Integer/byte work must match bit for bit; fp32
gradients within the stated relative tolerances."""
import ctypes as C

import numpy as np
import pytest

import openntc_b200 as ont
from openntc_b200 import _abi
from tests import helpers as H

pytestmark = pytest.mark.gpu

# tolerances (relative to the largest magnitude of the reference tensor)
TOL_FP32_VS_FP64 = 2e-4   # libontc fp32 path vs oracle fp64
TOL_TF32_VS_FP64 = 3e-2   # upstream cuBLAS TF32 path vs oracle fp64


@pytest.fixture(scope="module")
def ref_ctx_cls():
    from oracle.bindings import REF_SO, RefContext
    if not REF_SO.exists():
        pytest.skip(f"{REF_SO} not built")
    return RefContext


def rel_err(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    scale = max(np.abs(b).max(), 1e-30)
    return float(np.abs(a - b).max() / scale)


# ---------------------------------------------------------------- bit-exact kernels

def _pack_inputs(bits, rng):
    half = 1 << (bits - 1)
    delta = 2.0 / (1 << bits)
    lattice = (np.arange(-half - 2, half + 2) * delta).astype(np.float32)
    ties = ((np.arange(-half - 1, half + 1) + 0.5) / half).astype(np.float32)
    edges = np.array([-1.0, 1.0, 1.0 - delta, -1.0 - 1e-7, 1.0 + 1e-3, 0.0, -0.0, 1e-30, -1e-30], np.float32)
    rnd = rng.uniform(-1.3, 1.3, 8192).astype(np.float32)
    x = np.concatenate([lattice, ties, edges, rnd])
    pad = (-x.size) % (32 // bits)
    return np.concatenate([x, np.zeros(pad, np.float32)])


@pytest.mark.parametrize("bits", [2, 4])
def test_quantize_pack_bit_exact(lib, oracle, bits):
    x = _pack_inputs(bits, np.random.default_rng(bits))
    mine = np.zeros(x.size * bits // 32, np.uint32)
    assert lib.ontc_debug_quantize_pack(x.ctypes.data_as(C.c_void_p), x.size, bits, mine.ctypes.data_as(C.c_void_p)) == 0
    assert np.array_equal(mine, oracle.quantize_pack(x, bits))


@pytest.mark.parametrize("bits", [2, 4])
def test_quantize_pack_matches_upstream(lib, ref_ctx_cls, bits):
    x = _pack_inputs(bits, np.random.default_rng(10 + bits))
    ref = ref_ctx_cls(0)
    try:
        expect = ref.quantize_pack(x, bits)
    finally:
        ref.close()
    mine = np.zeros(x.size * bits // 32, np.uint32)
    lib.ontc_debug_quantize_pack(x.ctypes.data_as(C.c_void_p), x.size, bits, mine.ctypes.data_as(C.c_void_p))
    assert np.array_equal(mine, expect)


def _device_weights(lib):
    w = np.zeros(12, np.float32)
    assert lib.ontc_debug_lanczos_weights(w.ctypes.data_as(C.c_void_p)) == 0
    return w


def test_lanczos_weights_close_to_libm(lib, oracle):
    wd = _device_weights(lib)
    wh = oracle.lanczos_weights()
    ulp = np.abs(wd.view(np.int32).astype(np.int64) - wh.view(np.int32).astype(np.int64))
    # CUDA sinf (<= 2 ulp) vs glibc sinf (<= 1 ulp); the reductions themselves are checked bit-exact
    assert ulp.max() <= 4, (wd, wh)


def _images(rng):
    out = [rng.integers(0, 256, (64, 64, c), dtype=np.uint8) for c in (1, 2, 3, 4)]
    yy, xx = np.mgrid[0:128, 0:128]
    smooth = (127.5 + 120 * np.sin(xx / 7.0) * np.cos(yy / 11.0)).astype(np.uint8)
    out.append(np.stack([smooth, 255 - smooth, smooth // 2], -1))
    out.append(np.full((8, 8, 3), 255, np.uint8))
    out.append(np.zeros((4, 4, 1), np.uint8))
    return out


def test_lanczos_reduction_matches_oracle(lib, oracle):
    w = _device_weights(lib)
    for img in _images(np.random.default_rng(0)):
        d, c = img.shape[0], img.shape[2]
        mine = np.zeros((d // 2, d // 2, c), np.uint8)
        assert lib.ontc_debug_lanczos_down(img.ctypes.data_as(C.c_void_p), d, c, mine.ctypes.data_as(C.c_void_p)) == 0
        assert np.array_equal(mine, oracle.lanczos_down(img, w)), img.shape


def test_lanczos_reduction_matches_upstream(lib, ref_ctx_cls):
    ref = ref_ctx_cls(0)
    try:
        for img in _images(np.random.default_rng(1)):
            d, c = img.shape[0], img.shape[2]
            mine = np.zeros((d // 2, d // 2, c), np.uint8)
            lib.ontc_debug_lanczos_down(img.ctypes.data_as(C.c_void_p), d, c, mine.ctypes.data_as(C.c_void_p))
            assert np.array_equal(mine, ref.filter_lanczos(img)), img.shape
    finally:
        ref.close()


# ---------------------------------------------------------------- manifest + init vs upstream

@pytest.fixture(scope="module")
def set1024(materials):
    return materials(1024, 0, 9)


def test_mip_chain_and_package_match_upstream(set1024, ref_ctx_cls):
    ctx = H.new_context(ont.Profile.Bpp_0_5, set1024, min_dim=1024)
    ref = ref_ctx_cls(ont.Profile.Bpp_0_5)
    try:
        assert ref.load_manifest(set1024) == 0
        sh, rs = H.shape(ctx), ref.shape()
        assert sh["mips"] == rs["mips"] and sh["levels"] == rs["levels"] and sh["C"] == rs["C"]
        assert sh["mip_dim"] == rs["mip_dim"] and sh["g0"] == rs["g0"] and sh["g1"] == rs["g1"]
        td = ctx.get_texture_data()
        for s in range(td.tex_count):
            nch = td.channels[s]
            for m in range(sh["mips"]):
                d = sh["mip_dim"][m]
                mine = np.ctypeslib.as_array(td.mips[s][m], (d * d * nch,))
                assert np.array_equal(mine, ref.mip_host(s, m, d * d * nch)), (s, m)
        for m in range(sh["mips"]):
            d = sh["mip_dim"][m]
            assert np.array_equal(H.package(ctx, m, d * d * sh["C"]), ref.package(m, d * d * sh["C"])), m
    finally:
        ref.close()


def test_initial_state_matches_upstream(set1024, ref_ctx_cls):
    """Same std::mt19937(123) draws in the same order: identical fp32 latents and weights."""
    ctx = H.new_context(ont.Profile.Bpp_1_0, set1024, min_dim=1024)
    ref = ref_ctx_cls(ont.Profile.Bpp_1_0)
    try:
        assert ref.load_manifest(set1024) == 0
        ref.begin_training(0, 1)
        sh = H.shape(ctx)
        for l in range(sh["levels"]):
            assert np.array_equal(H.tensor(ctx, _abi.DBG_G0, l), ref.tensor(0, l)), l
            assert np.array_equal(H.tensor(ctx, _abi.DBG_G1, l), ref.tensor(1, l)), l
        W = H.tensor(ctx, _abi.DBG_W)
        F = sh["F"]
        assert np.array_equal(W[:64 * F], ref.tensor(10))
        assert np.array_equal(W[64 * F:64 * F + 4096], ref.tensor(11))
        assert np.array_equal(W[64 * F + 4096:], ref.tensor(12))
    finally:
        ref.close()


# ---------------------------------------------------------------- step-0 features and gradients

@pytest.fixture(scope="module")
def step0(set1024, ref_ctx_cls, oracle):
    """Both implementations run step 0 with the lock at step 0 (latents snapped, no noise).
    Returns the pieces the step-0 tests compare."""
    profile = ont.Profile.Bpp_0_5
    grids = 2
    ctx = H.new_context(profile, set1024, min_dim=1024, grids=grids, steps=100, lock_step=0)
    W_init = H.tensor(ctx, _abi.DBG_W)
    p = ctx.train(1)
    assert p.result == 0 and p.batches_complete == 1
    s = H.last_step(ctx)
    assert s.noise == 0 and s.step == 0
    ref = ref_ctx_cls(profile)
    assert ref.load_manifest(set1024) == 0
    ref.begin_training(0, grids, 100, 0)
    ref.train(1)
    yield dict(ctx=ctx, ref=ref, s=s, W_init=W_init, profile=profile, grids=grids)
    ref.close()


def test_step0_features_match_upstream(step0, oracle):
    ctx, ref, s = step0["ctx"], step0["ref"], step0["s"]
    sh = H.shape(ctx)
    F, mip = sh["F"], sh["mip_dim"][s.lod]
    T = min(mip, 256)
    B = step0["grids"] * T * T
    # upstream packs x_ as [F][B] with stride B (ntc_kernel.cu:128)
    X = ref.tensor(20, n=F * B).reshape(F, B)
    m, level = H.oracle_model(oracle, ctx, step0["profile"], s.lod)
    ost = oracle.step(T, [(s.ox[i], s.oy[i]) for i in range(s.n_grids)], 0, 0, s.lod / (sh["mips"] - 1))
    rng = np.random.default_rng(0)
    idx = np.unique(np.concatenate([np.arange(min(B, 4096)), rng.integers(0, B, 4096)]))
    for b in idx:
        g, r = divmod(int(b), T * T)
        x = (r % T + s.ox[g]) % mip
        y = (r // T + s.oy[g]) % mip
        assert np.array_equal(oracle.features(m, ost, x, y), X[:, b]), (b, x, y)


def _device_step0_grads(step0):
    ctx = step0["ctx"]
    H.set_tensor(ctx, _abi.DBG_W, 0, step0["W_init"])
    s = H.make_step(step0["s"].lod, [(step0["s"].ox[i], step0["s"].oy[i]) for i in range(step0["grids"])])
    loss = H.gradients(ctx, s)
    return loss, s


def test_step0_gradients_match_oracle(step0, oracle):
    ctx = step0["ctx"]
    loss, s = _device_step0_grads(step0)
    sh = H.shape(ctx)
    m, level = H.oracle_model(oracle, ctx, step0["profile"], s.lod)
    mip = sh["mip_dim"][s.lod]
    ost = oracle.step(min(mip, 256), [(s.ox[i], s.oy[i]) for i in range(s.n_grids)], 0, 0, s.lod / (sh["mips"] - 1))
    oloss, dW, dG0, dG1 = oracle.step_gradients(m, ost)
    assert abs(loss - oloss) <= 1e-5 * oloss
    assert rel_err(H.tensor(ctx, _abi.DBG_G0_GRAD, level), dG0) < TOL_FP32_VS_FP64
    assert rel_err(H.tensor(ctx, _abi.DBG_G1_GRAD, level), dG1) < TOL_FP32_VS_FP64
    dWd = H.tensor(ctx, _abi.DBG_W_GRAD)
    F = sh["F"]
    for lo, hi in [(0, 64 * F), (64 * F, 64 * F + 4096), (64 * F + 4096, 64 * F + 4096 + sh["C"] * 64)]:
        assert rel_err(dWd[lo:hi], dW[lo:hi]) < TOL_FP32_VS_FP64, (lo, hi)


def test_step0_gradients_match_upstream(step0, oracle):
    ctx, ref = step0["ctx"], step0["ref"]
    loss, s = _device_step0_grads(step0)
    sh = H.shape(ctx)
    level = ctx.feature_level_for_lod(s.lod)
    assert rel_err(H.tensor(ctx, _abi.DBG_G0_GRAD, level), ref.tensor(2, level)) < TOL_TF32_VS_FP64
    assert rel_err(H.tensor(ctx, _abi.DBG_G1_GRAD, level), ref.tensor(3, level)) < TOL_TF32_VS_FP64
    dWd = H.tensor(ctx, _abi.DBG_W_GRAD)
    F, Cn = sh["F"], sh["C"]
    assert rel_err(dWd[:64 * F], ref.tensor(13)) < TOL_TF32_VS_FP64
    assert rel_err(dWd[64 * F:64 * F + 4096], ref.tensor(14)) < TOL_TF32_VS_FP64
    assert rel_err(dWd[64 * F + 4096:64 * F + 4096 + Cn * 64], ref.tensor(15)[:Cn * 64]) < TOL_TF32_VS_FP64


# ---------------------------------------------------------------- one optimiser step

def test_adam_step_matches_oracle(materials, oracle):
    """A full training step before the lock (noise on): latents, moments and decoder after
    the step equal the oracle's Adam applied to the oracle's gradients."""
    profile = ont.Profile.Bpp_1_0
    ctx = H.new_context(profile, materials(256, 3, 9), min_dim=16, grids=2, steps=50)
    sh = H.shape(ctx)
    # warm the moments with a few steps so the update is not just lr*sign(g)
    ctx.train(3)
    before = {}
    for l in range(sh["levels"]):
        for k in (_abi.DBG_G0, _abi.DBG_G1, _abi.DBG_G0_M, _abi.DBG_G0_V, _abi.DBG_G1_M, _abi.DBG_G1_V):
            before[(k, l)] = H.tensor(ctx, k, l)
    for k in (_abi.DBG_W, _abi.DBG_W_M, _abi.DBG_W_V):
        before[(k, 0)] = H.tensor(ctx, k)
    ctx.train(1)
    s = H.last_step(ctx)
    assert s.noise == 1 and s.grid_update == 1
    level = s.level
    b0, b1, C0, C1, _ = H.PROFILE_SHAPES[profile]
    mip = sh["mip_dim"][s.lod]
    g0 = before[(_abi.DBG_G0, level)]
    g1 = before[(_abi.DBG_G1, level)]
    W = before[(_abi.DBG_W, 0)]
    target = H.package(ctx, s.lod, mip * mip * sh["C"])
    m = oracle.model(C0, C1, sh["F"], sh["C"], g0.reshape(sh["g0"][level], -1), g1.reshape(sh["g1"][level], -1), W,
                     target, mip, 2.0 / 2 ** b0, 2.0 / 2 ** b1)
    ost = oracle.step(min(mip, 256), [(s.ox[i], s.oy[i]) for i in range(s.n_grids)], 1, s.seed,
                      s.lod / (sh["mips"] - 1))
    _, dW, dG0, dG1 = oracle.step_gradients(m, ost)
    for (kp, km, kv, grad, delta) in [(_abi.DBG_G0, _abi.DBG_G0_M, _abi.DBG_G0_V, dG0, 2.0 / 2 ** b0),
                                      (_abi.DBG_G1, _abi.DBG_G1_M, _abi.DBG_G1_V, dG1, 2.0 / 2 ** b1)]:
        p, mm, vv = before[(kp, level)].copy(), before[(km, level)].copy(), before[(kv, level)].copy()
        g = grad.astype(np.float32)
        oracle.adam(p, mm, vv, g, s.lr_grid, s.gb1, s.gb2, 1, delta)
        assert rel_err(H.tensor(ctx, km, level), mm) < 1e-3
        assert rel_err(H.tensor(ctx, kv, level), vv) < 1e-3
        dp_dev = H.tensor(ctx, kp, level) - before[(kp, level)]
        dp_orc = p - before[(kp, level)]
        assert rel_err(dp_dev, dp_orc) < 5e-3
        # untouched latents still take the decayed-moment step, exactly as the oracle's
        untouched = grad == 0
        assert np.array_equal(H.tensor(ctx, kp, level)[untouched], p[untouched])
        assert not H.tensor(ctx, {_abi.DBG_G0: _abi.DBG_G0_GRAD, _abi.DBG_G1: _abi.DBG_G1_GRAD}[kp], level).any()
    p, mm, vv = W.copy(), before[(_abi.DBG_W_M, 0)].copy(), before[(_abi.DBG_W_V, 0)].copy()
    nupd = 64 * sh["F"] + 4096 + sh["C"] * 64
    oracle.adam(p[:nupd], mm[:nupd], vv[:nupd], dW[:nupd].astype(np.float32), s.lr_dec, s.b1, s.b2, 0, 0.0)
    assert rel_err(H.tensor(ctx, _abi.DBG_W)[:nupd] - W[:nupd], p[:nupd] - W[:nupd]) < 5e-3
    assert np.array_equal(H.tensor(ctx, _abi.DBG_W)[nupd:], W[nupd:])  # padded Wout rows never move


def test_bounded_wait_gives_up_and_leaves_the_device_usable(lib, oracle):
    """The tcgen05 kernels' mbarrier waits are bounded: a wait nothing completes gives up after
    its polls and is reported as a failure, and the device keeps working afterwards."""
    import time
    t0 = time.perf_counter()
    assert lib.ontc_debug_wait_timeout(5) == ont.Result.CudaFailure
    assert time.perf_counter() - t0 < 5.0
    assert lib.ontc_debug_wait_timeout(0) == ont.Result.InvalidState
    w = np.zeros(12, np.float32)
    assert lib.ontc_debug_lanczos_weights(w.ctypes.data_as(C.c_void_p)) == 0  # still usable
    assert np.abs(w - oracle.lanczos_weights()).max() < 1e-6

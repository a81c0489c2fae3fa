"""ctypes bindings of the parity checkers.  TEST INFRASTRUCTURE ONLY.

* `Oracle`  -- oracle/liboracle.so, the CPU restatement (ontc_oracle.h).
* `RefRuntime` -- oracle/_ref/libontc_ref_rt.so, upstream's CUDA-free runtime built from
  its sources (runs anywhere).
* `RefContext` -- oracle/_ref/libontc_ref.so, upstream's training library built from its
  sources (needs a GPU to run).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline / reference legs use this
module.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ORACLE_SO = HERE / "liboracle.so"
REF_RT_SO = HERE / "_ref" / "libontc_ref_rt.so"
REF_SO = HERE / "_ref" / "libontc_ref.so"

F32P = C.POINTER(C.c_float)
U8P = C.POINTER(C.c_uint8)
P = C.c_void_p


def _ptr(a: np.ndarray, t=C.c_void_p):
    return a.ctypes.data_as(t)


class OrcModel(C.Structure):
    _fields_ = [("C0", C.c_int32), ("C1", C.c_int32), ("F", C.c_int32), ("C", C.c_int32),
                ("g0_dim", C.c_int32), ("g1_dim", C.c_int32), ("mip_dim", C.c_int32),
                ("d0", C.c_float), ("d1", C.c_float),
                ("g0", F32P), ("g1", F32P), ("W", F32P), ("target", U8P)]


class OrcStep(C.Structure):
    _fields_ = [("tile_dim", C.c_int32), ("n_grids", C.c_int32), ("ox", C.c_int32 * 8), ("oy", C.c_int32 * 8),
                ("noise", C.c_int32), ("seed", C.c_uint32), ("norm_lod", C.c_float)]


def build_oracle():
    if not ORACLE_SO.exists():
        subprocess.run(["make", "-C", str(HERE), "liboracle.so"], check=True, capture_output=True)


class Oracle:
    def __init__(self):
        build_oracle()
        L = C.CDLL(str(ORACLE_SO))
        L.orc_texel_xy.argtypes = [C.POINTER(OrcStep), C.c_int32, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int32)]
        L.orc_noise.argtypes = [C.c_uint32, C.c_uint32, C.c_uint32, C.c_float]
        L.orc_noise.restype = C.c_float
        L.orc_features.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcStep), C.c_int32, C.c_int32, F32P]
        L.orc_step_gradients.argtypes = [C.POINTER(OrcModel), C.POINTER(OrcStep), P, P, P, C.c_int32]
        L.orc_step_gradients.restype = C.c_double
        L.orc_mip_sq_error.argtypes = [C.POINTER(OrcModel), C.c_float, C.c_int32, C.c_uint32, F32P, F32P, C.c_int32]
        L.orc_mip_sq_error.restype = C.c_double
        L.orc_adam.argtypes = [P, P, P, P, C.c_int64, C.c_float, C.c_float, C.c_float, C.c_int32, C.c_float]
        L.orc_quantize_grid.argtypes = [P, C.c_int64, C.c_int32, C.c_float]
        L.orc_quantize_pack.argtypes = [P, C.c_int64, C.c_int32, P]
        L.orc_lanczos_weights.argtypes = [P]
        L.orc_lanczos_down.argtypes = [P, C.c_int32, C.c_int32, P, P]
        L.orc_quantize_weights.argtypes = [P, C.c_int32, C.c_int32, C.c_float, P, P]
        L.orc_sample_material.argtypes = [C.c_int32, P, P, P, P, P, P, C.c_int64, P, C.c_int32]
        L.orc_decode_float.argtypes = [C.c_int32, P, P, P, P, C.c_int32, P, P, C.c_int64, P, C.c_int32]
        L.orc_screen_filter.argtypes = [P, C.c_int32, C.c_int32, C.c_int32, C.c_int32, C.c_float, C.c_int32, P, P, P,
                                        P, P]
        L.orc_decode_material.argtypes = [P, C.c_int64, C.c_int32, P, P]
        L.orc_check_div3.argtypes = [C.c_int32]
        L.orc_check_div3.restype = C.c_int64
        self.L = L
        self._keep = []

    # --- model / step helpers
    def model(self, C0, C1, F, Cout, g0, g1, W, target, mip_dim, d0, d1) -> OrcModel:
        g0 = np.ascontiguousarray(g0, np.float32)
        g1 = np.ascontiguousarray(g1, np.float32)
        W = np.ascontiguousarray(W, np.float32)
        target = np.ascontiguousarray(target, np.uint8)
        self._keep = [g0, g1, W, target]
        m = OrcModel(C0, C1, F, Cout, g0.shape[0], g1.shape[0], mip_dim, d0, d1,
                     _ptr(g0, F32P), _ptr(g1, F32P), _ptr(W, F32P), _ptr(target, U8P))
        return m

    @staticmethod
    def step(tile_dim, origins, noise=0, seed=0, norm_lod=0.0) -> OrcStep:
        s = OrcStep()
        s.tile_dim = tile_dim
        s.n_grids = len(origins)
        for i, (x, y) in enumerate(origins):
            s.ox[i], s.oy[i] = x, y
        s.noise, s.seed, s.norm_lod = noise, seed, norm_lod
        return s

    def texel_xy(self, s: OrcStep, mip_dim: int, b: int):
        x, y = C.c_int32(), C.c_int32()
        self.L.orc_texel_xy(C.byref(s), mip_dim, b, C.byref(x), C.byref(y))
        return x.value, y.value

    def features(self, m: OrcModel, s: OrcStep, x: int, y: int) -> np.ndarray:
        out = np.zeros(96, np.float32)
        self.L.orc_features(C.byref(m), C.byref(s), x, y, _ptr(out, F32P))
        return out[: m.F]

    def step_gradients(self, m: OrcModel, s: OrcStep, threads=8, latent_grads=True):
        nW = 64 * m.F + 64 * 64 + 16 * 64
        dW = np.zeros(nW, np.float64)
        dG0 = np.zeros(m.g0_dim * m.g0_dim * m.C0, np.float64) if latent_grads else None
        dG1 = np.zeros(m.g1_dim * m.g1_dim * m.C1, np.float64) if latent_grads else None
        loss = self.L.orc_step_gradients(C.byref(m), C.byref(s), _ptr(dW),
                                         _ptr(dG0) if dG0 is not None else None,
                                         _ptr(dG1) if dG1 is not None else None, threads)
        return loss, dW, dG0, dG1

    def mip_sq_error(self, m: OrcModel, norm_lod: float, noise=0, seed=0, threads=8):
        a0, a1 = C.c_float(), C.c_float()
        sq = self.L.orc_mip_sq_error(C.byref(m), norm_lod, noise, seed, C.byref(a0), C.byref(a1), threads)
        return sq, a0.value, a1.value

    def adam(self, p, m, v, g, lr, b1, b2, clamp, delta):
        for a in (p, m, v, g):
            assert a.dtype == np.float32 and a.flags.c_contiguous
        self.L.orc_adam(_ptr(p), _ptr(m), _ptr(v), _ptr(g), p.size, lr, b1, b2, clamp, delta)

    def quantize_grid(self, g: np.ndarray, bits: int, delta: float):
        self.L.orc_quantize_grid(_ptr(g), g.size, bits, delta)

    def quantize_pack(self, x: np.ndarray, bits: int) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros(x.size * bits // 32, np.uint32)
        self.L.orc_quantize_pack(_ptr(x), x.size, bits, _ptr(out))
        return out

    def lanczos_weights(self) -> np.ndarray:
        w = np.zeros(12, np.float32)
        self.L.orc_lanczos_weights(_ptr(w))
        return w

    def lanczos_down(self, img: np.ndarray, weights: np.ndarray) -> np.ndarray:
        img = np.ascontiguousarray(img, np.uint8)
        dim, c = img.shape[0], (img.shape[2] if img.ndim == 3 else 1)
        out = np.zeros((dim // 2, dim // 2, c), np.uint8)
        w = np.ascontiguousarray(weights, np.float32)
        self.L.orc_lanczos_down(_ptr(img), dim, c, _ptr(w), _ptr(out))
        return out

    def quantize_weights(self, Wf: np.ndarray, prescale: float):
        Wf = np.ascontiguousarray(Wf, np.float32)
        rows, cols = Wf.shape
        q = np.zeros(rows * cols // 4, np.uint32)
        s = np.zeros(rows, np.float32)
        self.L.orc_quantize_weights(_ptr(Wf), rows, cols, prescale, _ptr(q), _ptr(s))
        return q, s

    def sample_material(self, profile, g0, g1, decoder, consts_bytes, uv, lod, channels, threads=8):
        g0 = np.ascontiguousarray(np.concatenate([g0, np.zeros(4, np.uint32)]))
        g1 = np.ascontiguousarray(np.concatenate([g1, np.zeros(4, np.uint32)]))
        dec = np.ascontiguousarray(decoder, np.uint8)
        k = np.frombuffer(consts_bytes, np.uint8).copy()
        uv = np.ascontiguousarray(uv, np.float32)
        lod = np.ascontiguousarray(lod, np.int32)
        out = np.zeros((len(lod), channels), np.float32)
        self.L.orc_sample_material(profile, _ptr(g0), _ptr(g1), _ptr(dec), _ptr(k), _ptr(uv), _ptr(lod), len(lod),
                                   _ptr(out), threads)
        return out

    def screen_filter(self, img, dim, mip_count, noise_frame, discard_outside=False):
        """img float32 [h, w, 2] -> (uv [h*w, 2], lod [h*w], keep [h*w] bool, lod_ab [h*w], noise [h*w])."""
        img = np.ascontiguousarray(img, np.float32)
        h, w = img.shape[:2]
        n = h * w
        uv = np.zeros((n, 2), np.float32)
        lod = np.zeros(n, np.int32)
        keep = np.zeros(n, np.uint8)
        lod_ab = np.zeros(n, np.float32)
        noise = np.zeros(n, np.float32)
        self.L.orc_screen_filter(_ptr(img), w, h, dim, mip_count, noise_frame, int(bool(discard_outside)), _ptr(uv),
                                 _ptr(lod), _ptr(keep), _ptr(lod_ab), _ptr(noise))
        return uv, lod, keep.astype(bool), lod_ab, noise

    def decode_material(self, channels, semantics):
        """channels float32 [n, C], semantics [C] -> float32 [n, 18] (the last word is `present`)."""
        channels = np.ascontiguousarray(channels, np.float32)
        sem = np.zeros(16, np.uint32)
        sem[:len(semantics)] = semantics
        out = np.zeros((len(channels), 18), np.float32)
        self.L.orc_decode_material(_ptr(channels), len(channels), channels.shape[1], _ptr(sem), _ptr(out))
        return out

    def decode_float(self, profile, g0, g1, consts_bytes, W, channels, uv, lod, threads=8):
        g0 = np.ascontiguousarray(np.concatenate([g0, np.zeros(4, np.uint32)]))
        g1 = np.ascontiguousarray(np.concatenate([g1, np.zeros(4, np.uint32)]))
        k = np.frombuffer(consts_bytes, np.uint8).copy()
        W = np.ascontiguousarray(W, np.float32)
        uv = np.ascontiguousarray(uv, np.float32)
        lod = np.ascontiguousarray(lod, np.int32)
        out = np.zeros((len(lod), channels), np.float64)
        self.L.orc_decode_float(profile, _ptr(g0), _ptr(g1), _ptr(k), _ptr(W), channels, _ptr(uv), _ptr(lod),
                                len(lod), _ptr(out), threads)
        return out


class RefRuntime:
    """Upstream's openntc_runtime.cpp (Dump / Load / FillNTCConstants / tables)."""

    def __init__(self):
        if not REF_RT_SO.exists():
            raise FileNotFoundError(REF_RT_SO)
        L = C.CDLL(str(REF_RT_SO))
        L.ref_rt_dump.argtypes = [C.c_char_p, P]
        L.ref_rt_load.argtypes = [C.c_char_p, C.POINTER(P), P]
        L.ref_rt_free.argtypes = [P]
        L.ref_rt_fill_constants.argtypes = [P, P]
        L.ref_rt_semantic_from_name.argtypes = [C.c_char_p]
        L.ref_rt_semantic_to_string.argtypes = [C.c_int]
        L.ref_rt_semantic_to_string.restype = C.c_char_p
        L.ref_rt_channel_count.argtypes = [C.c_int]
        L.ref_rt_profile_to_string.argtypes = [C.c_int]
        L.ref_rt_profile_to_string.restype = C.c_char_p
        L.ref_rt_profile_from_string.argtypes = [C.c_char_p, C.POINTER(C.c_int)]
        self.L = L


class RefContext:
    """Upstream's openntc::Context (libopenntc.cpp) through oracle/ref_harness.cpp."""

    SHAPE_LEN = 32

    def __init__(self, profile: int):
        if not REF_SO.exists():
            raise FileNotFoundError(REF_SO)
        L = C.CDLL(str(REF_SO))
        L.ref_create.argtypes = [C.c_int, C.POINTER(C.c_int)]
        L.ref_create.restype = P
        L.ref_destroy.argtypes = [P]
        L.ref_load_manifest.argtypes = [P, C.c_char_p]
        L.ref_begin_training.argtypes = [P, C.c_int, C.c_int, C.c_int, C.c_int]
        L.ref_train.argtypes = [P, C.c_int, P]
        L.ref_time_train.argtypes = [P, C.c_int, C.POINTER(C.c_float), P]
        L.ref_eval.argtypes = [P, P]
        L.ref_calibrate.argtypes = [P, P]
        L.ref_get_compressed.argtypes = [P, P]
        L.ref_shape.argtypes = [P, P]
        L.ref_tensor.argtypes = [P, C.c_int, C.c_int, P, C.c_longlong, C.c_int]
        L.ref_tensor.restype = C.c_longlong
        L.ref_package.argtypes = [P, C.c_int, P]
        L.ref_mip_host.argtypes = [P, C.c_int, C.c_int]
        L.ref_mip_host.restype = C.POINTER(C.c_uint8)
        L.ref_decoder_host.argtypes = [P, C.POINTER(C.c_longlong)]
        L.ref_decoder_host.restype = C.POINTER(C.c_uint8)
        L.ref_quantize_pack.argtypes = [P, C.c_longlong, C.c_int, P]
        L.ref_filter_lanczos.argtypes = [P, C.c_int, C.c_int, P]
        self.L = L
        r = C.c_int()
        self.h = L.ref_create(profile, C.byref(r))
        self.init_result = r.value

    def close(self):
        if self.h:
            self.L.ref_destroy(self.h)
            self.h = None

    def load_manifest(self, path) -> int:
        return self.L.ref_load_manifest(self.h, str(path).encode())

    def begin_training(self, quality, grids, steps=0, lock=-1):
        self.L.ref_begin_training(self.h, quality, grids, steps, lock)

    def train(self, n):
        p = (C.c_int32 * 4)()
        self.L.ref_train(self.h, n, p)
        return list(p)

    def time_train(self, n):
        p = (C.c_int32 * 4)()
        ms = C.c_float()
        err = self.L.ref_time_train(self.h, n, C.byref(ms), p)
        return ms.value, list(p), err

    def eval(self):
        o = (C.c_double * 2)()
        self.L.ref_eval(self.h, o)
        return o[0], o[1]

    def shape(self):
        o = np.zeros(self.SHAPE_LEN, np.int32)
        self.L.ref_shape(self.h, _ptr(o))
        return {"levels": int(o[0]), "mips": int(o[1]), "F": int(o[2]), "Fp": int(o[3]), "C": int(o[4]),
                "g0": [int(v) for v in o[5:11]], "g1": [int(v) for v in o[11:17]],
                "mip_dim": [int(v) for v in o[17:29]], "batch_i": int(o[29]), "lock_i": int(o[30]),
                "batch_count": int(o[31])}

    def tensor(self, which: int, level: int = 0, n: int | None = None) -> np.ndarray:
        total = self.L.ref_tensor(self.h, which, level, None, 0, 0)
        n = total if n is None else n
        out = np.zeros(n, np.float32)
        got = self.L.ref_tensor(self.h, which, level, _ptr(out), n, 0)
        assert got == n, (which, level, got, n)
        return out

    def set_tensor(self, which: int, level: int, data: np.ndarray):
        data = np.ascontiguousarray(data, np.float32)
        got = self.L.ref_tensor(self.h, which, level, _ptr(data), data.size, 1)
        assert got == data.size

    def package(self, mip: int, size: int) -> np.ndarray:
        out = np.zeros(size, np.uint8)
        assert self.L.ref_package(self.h, mip, _ptr(out)) == 0
        return out

    def mip_host(self, source: int, mip: int, size: int) -> np.ndarray:
        p = self.L.ref_mip_host(self.h, source, mip)
        return np.ctypeslib.as_array(p, shape=(size,)).copy()

    def compressed(self):
        """Upstream's GetCompressedData() (libopenntc.cpp:1055-1101) as the layout-identical
        ontc_compressed_data mirror; its pointers borrow upstream's host buffers."""
        from openntc_b200 import _abi
        cd = _abi.CompressedData()
        self.L.ref_get_compressed(self.h, C.byref(cd))
        return cd

    def decoder(self) -> np.ndarray:
        n = C.c_longlong()
        p = self.L.ref_decoder_host(self.h, C.byref(n))
        return np.ctypeslib.as_array(p, shape=(n.value,)).copy()

    def quantize_pack(self, x: np.ndarray, bits: int) -> np.ndarray:
        x = np.ascontiguousarray(x, np.float32)
        out = np.zeros(x.size * bits // 32, np.uint32)
        assert self.L.ref_quantize_pack(_ptr(x), x.size, bits, _ptr(out)) == 0
        return out

    def filter_lanczos(self, img: np.ndarray) -> np.ndarray:
        img = np.ascontiguousarray(img, np.uint8)
        dim, c = img.shape[0], img.shape[2]
        out = np.zeros((dim // 2, dim // 2, c), np.uint8)
        assert self.L.ref_filter_lanczos(_ptr(img), dim, c, _ptr(out)) == 0
        return out


# upstream tensor selectors of ref_harness.cpp:tensor_ptr
REF_G0, REF_G1, REF_DG0, REF_DG1 = 0, 1, 2, 3
REF_W0, REF_W1, REF_WOUT, REF_DW0, REF_DW1, REF_DWOUT = 10, 11, 12, 13, 14, 15
REF_X, REF_DX, REF_Y = 20, 21, 22

"""The C ABI of libontc.so: it loads, exports every declared symbol, and its structs have
upstream's layout (no GPU needed)."""
import ctypes as C
import subprocess

import pytest

import openntc_b200 as ont
from openntc_b200 import _abi
from tests.conftest import HAS_GPU, ROOT

HEADERS = [ROOT / "include" / "ontc.h", ROOT / "include" / "ontc_debug.h"]


def test_library_exports_every_declared_symbol(lib):
    declared = []
    for h in HEADERS:
        declared += _abi.declared_symbols(h)
    assert len(declared) >= 38
    missing = [s for s in declared if not hasattr(lib, s)]
    assert not missing, missing
    # every declared symbol has a ctypes signature in the mirror
    assert not [s for s in declared if s not in _abi.SIGNATURES], [s for s in declared if s not in _abi.SIGNATURES]


def _c_layout(tmp_path):
    """sizeof/offsetof of the public structs as the C compiler lays them out."""
    src = tmp_path / "layout.c"
    fields = {
        "ontc_compressed_data": [f for f, _ in _abi.CompressedData._fields_],
        "ontc_constants": [f for f, _ in _abi.Constants._fields_],
        "ontc_train_progress": [f for f, _ in _abi.TrainProgress._fields_],
        "ontc_eval_results": [f for f, _ in _abi.EvalResults._fields_],
        "ontc_texture_data": [f for f, _ in _abi.TextureData._fields_],
        "ontc_train_options": [f for f, _ in _abi.TrainOptions._fields_],
        "ontc_calibration": [f for f, _ in _abi.Calibration._fields_],
        "ontc_debug_step": [f for f, _ in _abi.DebugStep._fields_],
    }
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ontc_debug.h"', "int main(void){"]
    for s, fs in fields.items():
        lines.append(f'printf("{s} %zu\\n", sizeof({s}));')
        for f in fs:
            lines.append(f'printf("{s}.{f} %zu\\n", offsetof({s}, {f}));')
    lines.append("return 0;}")
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return dict((k, int(v)) for k, v in (l.split() for l in out.splitlines()))


def test_struct_layouts_match_c(tmp_path):
    lay = _c_layout(tmp_path)
    for name, cls in [("ontc_compressed_data", _abi.CompressedData), ("ontc_constants", _abi.Constants),
                      ("ontc_train_progress", _abi.TrainProgress), ("ontc_eval_results", _abi.EvalResults),
                      ("ontc_texture_data", _abi.TextureData), ("ontc_train_options", _abi.TrainOptions),
                      ("ontc_calibration", _abi.Calibration), ("ontc_debug_step", _abi.DebugStep)]:
        assert lay[name] == C.sizeof(cls), name
        for f, _ in cls._fields_:
            assert lay[f"{name}.{f}"] == getattr(cls, f).offset, f"{name}.{f}"
    assert lay["ontc_constants"] == 240  # openntc_runtime.h:89


def test_struct_layouts_match_upstream(ref_rt):
    assert ref_rt.L.ref_rt_sizeof_compressed() == C.sizeof(_abi.CompressedData)
    assert ref_rt.L.ref_rt_sizeof_constants() == C.sizeof(_abi.Constants)


def test_steps_for_quality():
    # libopenntc.cpp:428-443
    assert [ont.steps_for_quality(q) for q in range(4)] == [30000, 120000, 240000, 480000]
    assert ont.steps_for_quality(99) == 30000


@pytest.mark.skipif(HAS_GPU, reason="checks the no-GPU path")
def test_init_without_gpu_fails_loudly():
    ctx = ont.Context()
    assert ctx.init(ont.Profile.Bpp_0_5) == ont.Result.CudaFailure


def test_uninitialised_context_rejects_training():
    ctx = ont.Context()
    p = ctx.train(10)
    assert p.phase == ont.TrainPhase.TrainError and p.result == ont.Result.InvalidState
    r = ctx.eval()
    assert r.mse == 0.0 and ctx.get_last_error() == ont.Result.InvalidState
    assert ctx.get_mip_dim(0) == 0


def test_product_path_refuses_to_run_without_library(tmp_path, monkeypatch):
    import openntc_b200
    monkeypatch.setattr(openntc_b200, "_lib", None)
    monkeypatch.setattr(openntc_b200, "LIB_PATH", tmp_path / "missing.so")
    with pytest.raises(RuntimeError):
        openntc_b200.load()


def test_disjoint_cover_keeps_the_union(lib):
    """The deferred optimiser's footprint cover: disjoint rectangles, same union as the input."""
    import numpy as np
    rng = np.random.default_rng(7)
    for case in range(300):
        n = int(rng.integers(0, 17))
        dim = 64
        x0 = rng.integers(0, dim, n); y0 = rng.integers(0, dim, n)
        x1 = np.minimum(dim, x0 + rng.integers(1, 40, n)); y1 = np.minimum(dim, y0 + rng.integers(1, 40, n))
        inp = np.stack([x0, y0, x1, y1], 1).astype(np.int32).copy()
        out = np.zeros((256, 4), np.int32)
        m = lib.ontc_debug_disjoint_cover(inp.ctypes.data, n, out.ctypes.data, 256)
        assert m >= 0
        want = np.zeros((dim, dim), np.int32)
        for a, b, c, d in inp:
            want[b:d, a:c] = 1
        got = np.zeros((dim, dim), np.int32)
        for a, b, c, d in out[:m]:
            assert a < c and b < d
            got[b:d, a:c] += 1
        assert np.array_equal(got, want), case  # covered exactly once where the union is
    one = np.array([[0, 0, 8, 8], [4, 4, 12, 12], [20, 0, 24, 4]], np.int32)
    out = np.zeros((4, 4), np.int32)
    assert lib.ontc_debug_disjoint_cover(one.ctypes.data, 3, out.ctypes.data, 2) == -1


def test_footprint_intersection_and_difference_covers(lib):
    """Consecutive steps' footprints split into shared cells and cells of one step only: each
    cover is disjoint and selects exactly the cells of A in (op 1) or outside (op 2) B."""
    import numpy as np
    rng = np.random.default_rng(11)
    dim = 64

    def rects(n):
        x0 = rng.integers(0, dim, n); y0 = rng.integers(0, dim, n)
        x1 = np.minimum(dim, x0 + rng.integers(1, 40, n)); y1 = np.minimum(dim, y0 + rng.integers(1, 40, n))
        return np.stack([x0, y0, x1, y1], 1).astype(np.int32).copy()

    def grid(rs):
        g = np.zeros((dim, dim), bool)
        for a, b, c, d in rs:
            g[b:d, a:c] = True
        return g

    for case in range(300):
        A, B = rects(int(rng.integers(0, 9))), rects(int(rng.integers(0, 9)))
        for op, want in ((1, grid(A) & grid(B)), (2, grid(A) & ~grid(B))):
            out = np.zeros((512, 4), np.int32)
            m = lib.ontc_debug_cover_op(A.ctypes.data, len(A), B.ctypes.data, len(B), op, out.ctypes.data, 512)
            assert m >= 0
            got = np.zeros((dim, dim), np.int32)
            for a, b, c, d in out[:m]:
                assert a < c and b < d
                got[b:d, a:c] += 1
            assert np.array_equal(got, want.astype(np.int32)), (case, op)
    assert lib.ontc_debug_cover_op(A.ctypes.data, len(A), B.ctypes.data, len(B), 0, out.ctypes.data, 512) == -1

"""Host-side error paths, with the failure made on the host (no GPU fault):

* malformed manifests: libontc's ontc_load_manifest must return what upstream's own
  Context::LoadManifest returns on the same file (libopenntc.cpp:1125-1336: FileNotFound,
  InvalidManifest, InvalidDimension), case by case;
* an out-of-memory cudaMalloc at every device allocation point of a whole context lifetime
  (ontc_debug_fail_device_alloc): the call that hit it reports the failure (a Result, or
  TrainError progress and GetLastError, as upstream's OPENNTC_CUDA_CHECK paths do,
  libopenntc.cpp:17-30, :506-527), nothing later runs on the missing buffer, the context can
  be destroyed, and the device's free memory is back where it started.
"""
import json

import numpy as np
import pytest

import openntc_b200 as ont

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def ref_cls():
    from oracle.bindings import REF_SO, RefContext
    if not REF_SO.exists():
        pytest.skip(f"{REF_SO} not built")
    return RefContext


def _manifest_cases(base, tmp):
    """(name, manifest text or None for a missing file) built around a valid 1024^2 set."""
    good = json.loads(base.read_text())
    tex = good["textures"]
    small = tmp / "small.ppm"
    small.write_bytes(b"P6\n512 512\n255\n" + bytes(512 * 512 * 3))
    wide = tmp / "wide.ppm"
    wide.write_bytes(b"P6\n1024 512\n255\n" + bytes(1024 * 512 * 3))
    garbage = tmp / "garbage.png"
    garbage.write_bytes(b"\x89PNG\r\n\x1a\n not really")

    def m(**kw):
        d = dict(good)
        d.update(kw)
        return json.dumps({k: v for k, v in d.items() if v is not None})

    def with_tex(t):
        return m(textures=t)

    cases = [
        ("valid", m()),
        ("width_only", json.dumps({"width": 1024, "textures": tex})),
        ("height_only", json.dumps({"height": 1024, "textures": tex})),
        ("missing_file", None),
        ("not_json", "{ this is not json"),
        ("no_textures", json.dumps({"width": 1024, "height": 1024})),
        ("no_size", json.dumps({"textures": tex})),
        ("not_square", m(height=512)),
        ("below_min", m(width=512, height=512)),
        ("above_max", m(width=16384, height=16384)),
        ("not_pow2", m(width=1536, height=1536)),
        ("no_semantics", with_tex([{"fileName": tex[0]["fileName"]}] + tex[1:])),
        ("semantics_not_object", with_tex([{"fileName": tex[0]["fileName"], "semantics": "Albedo"}] + tex[1:])),
        ("no_file_name", with_tex([{"semantics": {"Albedo": "RGB"}}] + tex[1:])),
        ("file_name_not_string", with_tex([{"fileName": 7, "semantics": {"Albedo": "RGB"}}] + tex[1:])),
        ("channels_not_string", with_tex([dict(tex[0], semantics={"Albedo": 3})] + tex[1:])),
        ("wrong_channel_count", with_tex([dict(tex[0], semantics={"Albedo": "RG"})] + tex[1:])),
        ("channels_out_of_order", with_tex([dict(tex[0], semantics={"Albedo": "BGR"})] + tex[1:])),
        ("channels_repeated", with_tex([dict(tex[0], semantics={"Albedo": "RRG"})] + tex[1:])),
        ("too_many_channel_letters", with_tex([dict(tex[0], semantics={"Albedo": "RGBAR"})] + tex[1:])),
        ("empty_channels", with_tex([dict(tex[0], semantics={"Albedo": ""})] + tex[1:])),
        ("bad_channel_letter", with_tex([dict(tex[0], semantics={"Albedo": "RGX"})] + tex[1:])),
        ("unknown_semantic_alone", with_tex([dict(tex[0], semantics={"Sparkle": "R"})])),
        # not run through upstream: an unknown name is Semantic::None with a channel count of -1
        # (openntc_runtime.cpp:89), which beside valid sources passes the total-channel check
        # (libopenntc.cpp:1188) and reaches allocations and kernel launches with that count
        ("unknown_semantic_beside", with_tex(tex + [dict(tex[0], semantics={"Sparkle": "R"})])),
        ("no_channels_at_all", with_tex([])),
        ("seventeen_channels", with_tex([dict(tex[0], semantics={s: "RGB"}) for s in
                                         ("Albedo", "Normal", "Specular", "Albedo", "Normal")]
                                        + [dict(tex[0], semantics={"Roughness": "R", "Metallic": "G"})])),
        ("sixteen_channels", with_tex([dict(tex[0], semantics={s: "RGB"}) for s in
                                       ("Albedo", "Normal", "Specular", "Albedo", "Normal")]
                                      + [dict(tex[0], semantics={"Roughness": "R"})])),
        ("image_missing", with_tex([dict(tex[0], fileName=str(tmp / "nope.ppm"))] + tex[1:])),
        ("image_wrong_size", with_tex([dict(tex[0], fileName=str(small))] + tex[1:])),
        ("image_not_square", with_tex([dict(tex[0], fileName=str(wide))] + tex[1:])),
        ("image_undecodable", with_tex([dict(tex[0], fileName=str(garbage))] + tex[1:])),
    ]
    return cases


# cases upstream handles with undefined behaviour: libontc's result instead
NOT_UPSTREAM = {"unknown_semantic_beside": "InvalidManifest"}


def test_malformed_manifests_match_upstream(materials, ref_cls, tmp_path):
    base = materials(1024, 13, 9)
    ctx = ont.Context()
    assert ctx.init(ont.Profile.Bpp_0_5) == ont.Result.Success
    ref = ref_cls(ont.Profile.Bpp_0_5)
    results = {}
    try:
        for name, text in _manifest_cases(base, tmp_path):
            path = tmp_path / f"{name}.json"
            if text is not None:
                path.write_text(text)
            mine = int(ctx.load_manifest(path))
            if name in NOT_UPSTREAM:
                results[name] = (ont.Result(mine).name, NOT_UPSTREAM[name])
                continue
            theirs = ref.load_manifest(path)
            results[name] = (ont.Result(mine).name, ont.Result(theirs).name)
    finally:
        ref.close()
        ctx.destroy()
    print(results)
    assert results["valid"] == ("Success", "Success") and results["sixteen_channels"] == ("Success", "Success")
    assert {n for n, (a, b) in results.items() if a != "Success"} >= {
        "missing_file", "not_json", "not_square", "below_min", "not_pow2", "image_missing", "image_wrong_size"}
    bad = {n: r for n, r in results.items() if r[0] != r[1]}
    assert not bad, bad


def _lifetime(manifest, calls):
    """One context from init to destroy; returns the first failure as (call, detail)."""
    ctx = ont.Context()
    try:
        r = ctx.init(ont.Profile.Bpp_2_25)
        calls.append(("init", int(r)))
        if r != ont.Result.Success:
            return "init", int(r)
        assert ctx.set_min_dimension(16) == ont.Result.Success
        r = ctx.load_manifest(manifest)
        calls.append(("load_manifest", int(r)))
        if r != ont.Result.Success:
            # nothing of the manifest is held and the context refuses to train
            p = ctx.train(1)
            assert p.phase == ont.TrainPhase.TrainError and p.result == ont.Result.InvalidState
            return "load_manifest", int(r)
        try:  # ontc_begin_training, then ontc_set_train_options (its own step-loss buffer)
            ctx.begin_training(ont.Quality.Low, 2, steps=40, precision=ont.Precision.BF16)
        except RuntimeError:
            pass
        if ctx.get_last_error() != ont.Result.Success:
            p = ctx.train(1)  # must not run on the missing step-loss buffer
            assert p.phase == ont.TrainPhase.TrainError and p.result == ont.Result.InvalidState, p
            return "begin_training", int(ctx.get_last_error())
        for n in (5, 40):
            p = ctx.train(n)
            if p.result != ont.Result.Success:
                assert p.phase == ont.TrainPhase.TrainError
                return "train", int(p.result)
        assert p.phase == ont.TrainPhase.TrainComplete
        e = ctx.eval()
        if ctx.get_last_error() != ont.Result.Success:
            return "eval", int(ctx.get_last_error())
        assert np.isfinite(e.psnr)
        e = ctx.eval_decoded()
        if ctx.get_last_error() != ont.Result.Success:
            return "eval_decoded", int(ctx.get_last_error())
        return None
    finally:
        ctx.destroy()


def test_every_device_allocation_failure_is_reported_and_leaks_nothing(materials, lib):
    import torch
    manifest = materials(256, 14, 9)
    lib.ontc_debug_fail_device_alloc(0)
    assert _lifetime(manifest, []) is None  # warm-up: driver-side state settles
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    start = lib.ontc_debug_fail_device_alloc(0)
    assert _lifetime(manifest, []) is None
    total = lib.ontc_debug_fail_device_alloc(0) - start
    assert total > 20, total
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    seen = {}
    for n in range(1, total + 1):
        lib.ontc_debug_fail_device_alloc(n)
        calls = []
        failed = _lifetime(manifest, calls)
        lib.ontc_debug_fail_device_alloc(0)
        assert failed is not None, (n, calls)
        where, code = failed
        assert code in (ont.Result.AllocationFailure, ont.Result.CudaFailure), (n, where, code)
        seen.setdefault(where, []).append(n)
        torch.cuda.synchronize()
        assert torch.cuda.mem_get_info()[0] == free0, (n, where)
    print({k: (len(v), v[0], v[-1]) for k, v in seen.items()})
    assert {"init", "load_manifest", "begin_training"} <= set(seen)
    # the context works again once allocations succeed
    assert _lifetime(manifest, []) is None

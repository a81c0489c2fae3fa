"""ONTC container, constant buffer and name tables against upstream's runtime
(libopenntc/openntc_runtime.cpp), no GPU needed."""
import ctypes as C
import json
import random
import struct

import numpy as np
import pytest

import openntc_b200 as ont
from openntc_b200 import _abi
from tests.conftest import ROOT
from tests.golden.cases import Case, corruptions

GOLD = ROOT / "tests" / "golden" / "runtime"


@pytest.mark.parametrize("seed", range(12))
def test_dump_matches_golden_bytes(seed, tmp_path):
    c = Case(seed)
    p = tmp_path / "x.ntc"
    assert ont.dump(p, c.data) == ont.Result.Success
    assert p.read_bytes() == (GOLD / f"case_{seed}.ntc").read_bytes()


def test_dump_matches_upstream_live(ref_rt, tmp_path):
    """Randomised: upstream's Dump and ours produce identical bytes (JSON float format included)."""
    for seed in range(1000, 1400):
        c = Case(seed)
        a, b = tmp_path / "a.ntc", tmp_path / "b.ntc"
        assert ont.dump(a, c.data) == 0
        assert ref_rt.L.ref_rt_dump(str(b).encode(), C.byref(c.data)) == 0
        assert a.read_bytes() == b.read_bytes(), seed


def test_json_float_format_matches_upstream(ref_rt, tmp_path):
    """Edge floats through the calibration block: subnormals, powers of ten, ties."""
    vals = [0.0, -0.0, 1e-45, 1.17549435e-38, 3.4028235e38, 1e-5, 1e-4, 0.001, 123456.79, 1e15, 1e16, 9.999999e14,
            0.1, 0.2, 0.3, 1.0 / 3.0, 2.0 / 3.0, 799.6094360351562, 1e21, 5e-324]
    rng = random.Random(7)
    vals += [struct.unpack("f", struct.pack("I", rng.getrandbits(32) & 0x7F7FFFFF))[0] for _ in range(400)]
    c = Case(3)
    for i in range(0, len(vals), 4):
        quad = (vals[i:i + 4] + [1.0] * 4)[:4]
        c.data.caldata.max_abs_a1, c.data.caldata.max_abs_a2, c.data.caldata.s_a1, c.data.caldata.s_a2 = quad
        a, b = tmp_path / "a.ntc", tmp_path / "b.ntc"
        ont.dump(a, c.data)
        ref_rt.L.ref_rt_dump(str(b).encode(), C.byref(c.data))
        assert a.read_bytes() == b.read_bytes(), quad


def _load(path):
    r, fd = ont.load_file(path)
    return r, fd


@pytest.mark.parametrize("seed", range(12))
def test_load_roundtrip(seed, tmp_path):
    c = Case(seed)
    r, fd = _load(GOLD / f"case_{seed}.ntc")
    assert r == ont.Result.Success
    d = fd.data
    for f in ("dim", "mip_count", "level_count", "channel_count", "profile", "g0_bits_per_channel",
              "g1_bits_per_channel", "g0_channels", "g1_channels", "decoder_size"):
        assert getattr(d, f) == getattr(c.data, f), f
    for i in range(c.data.level_count):
        assert d.g0_size[i] == c.data.g0_size[i] and d.g1_size[i] == c.data.g1_size[i]
        assert d.g0_grid_dim[i] == c.data.g0_grid_dim[i]
        a = np.ctypeslib.as_array(C.cast(d.g0[i], C.POINTER(C.c_uint8)), (d.g0_size[i],))
        b = np.ctypeslib.as_array(C.cast(c.data.g0[i], C.POINTER(C.c_uint8)), (d.g0_size[i],))
        assert np.array_equal(a, b)
    # pyramids are repacked contiguously (openntc_runtime.cpp:433-453)
    assert d.g0_offset[0] == 0
    for i in range(1, d.level_count):
        assert d.g0_offset[i] == d.g0_offset[i - 1] + d.g0_size[i - 1]
    assert d.g0_total_size == sum(d.g0_size[i] for i in range(d.level_count))
    for f in ("max_abs_a1", "max_abs_a2", "s_a1", "s_a2"):
        assert np.float32(getattr(d.caldata, f)) == np.float32(getattr(c.data.caldata, f))
    # dump(load(x)) == x
    p = tmp_path / "re.ntc"
    assert ont.dump(p, d) == 0
    assert p.read_bytes() == (GOLD / f"case_{seed}.ntc").read_bytes()


def test_load_matches_upstream_fields(ref_rt):
    for seed in range(12):
        path = GOLD / f"case_{seed}.ntc"
        r, fd = _load(path)
        h = C.c_void_p()
        ref_cd = _abi.CompressedData()
        rr = ref_rt.L.ref_rt_load(str(path).encode(), C.byref(h), C.byref(ref_cd))
        assert r == rr == 0
        # upstream leaves entries past level_count / channel_count uninitialised
        # (FileData::data_ is never zeroed, openntc_runtime.cpp:458), so only defined ones compare
        L, Cn = fd.data.level_count, fd.data.channel_count
        for f, _ in _abi.CompressedData._fields_:
            if f in ("g0", "g1", "decoder", "caldata"):
                continue
            va, vb = getattr(fd.data, f), getattr(ref_cd, f)
            if hasattr(va, "__len__"):
                n = Cn if f == "channel_semantics" else L
                assert list(va)[:n] == list(vb)[:n], f
            else:
                assert va == vb, f
        ref_rt.L.ref_rt_free(h)


def test_load_error_codes_match_upstream(tmp_path):
    expected = json.loads((GOLD / "load_results.json").read_text())
    raw = (GOLD / "case_0.ntc").read_bytes()
    for name, blob in corruptions(raw).items():
        p = tmp_path / f"{name}.ntc"
        p.write_bytes(blob)
        r, _ = _load(p)
        assert int(r) == expected[name], name
    r, _ = _load(tmp_path / "does_not_exist.ntc")
    assert r == ont.Result.FileNotFound


def test_fill_constants_matches_upstream(ref_rt):
    for seed in range(12):
        c = Case(seed)
        mine = ont.fill_constants(c.data)
        ref = (C.c_uint8 * 240)()
        ref_rt.L.ref_rt_fill_constants(C.byref(c.data), ref)
        assert bytes(mine) == bytes(ref), seed


def test_name_tables_match_upstream(ref_rt):
    names = ["Albedo", "Diffuse", "Alpha", "Mask", "AlphaMask", "Displ", "Displacement", "Emissive", "Emission",
             "Glossiness", "Gloss", "Metalness", "Metallic", "Normal", "Occlusion", "AO", "AmbientOcclusion",
             "Roughness", "SpecularColor", "Specular", "Transmission", "albedo", "", "Bogus", "None"]
    for n in names:
        assert ont.semantic_from_name(n) == ref_rt.L.ref_rt_semantic_from_name(n.encode()), n
    for s in range(-1, 14):
        assert ont.semantic_to_string(s).encode() == ref_rt.L.ref_rt_semantic_to_string(s), s
    for s in range(0, 13):
        assert ont.channel_count_for_semantic(s) == ref_rt.L.ref_rt_channel_count(s), s
    for p in range(-1, 5):
        assert ont.profile_to_string(p).encode() == ref_rt.L.ref_rt_profile_to_string(p)
    for s in ["bpp_0_2", "bpp_0_5", "bpp_1_0", "bpp_2_25", "bpp_1", ""]:
        o = C.c_int(-1)
        ok = ref_rt.L.ref_rt_profile_from_string(s.encode(), C.byref(o))
        mine = ont.profile_from_string(s)
        assert (mine is not None) == bool(ok) and (mine is None or mine == o.value), s

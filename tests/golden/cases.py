"""Deterministic CompressedData cases for the ONTC container tests (shared by the fixture
generator and the tests)."""
from __future__ import annotations

import ctypes as C
import random
import struct

import numpy as np

from openntc_b200 import _abi


class Case:
    """Owns the blob memory a CompressedData points into."""

    def __init__(self, seed: int):
        r = random.Random(seed)
        self.keep = []
        d = _abi.CompressedData()
        levels = r.randint(1, 6)
        d.level_count = levels
        d.mip_count = r.randint(1, 12)
        d.dim = 1 << r.randint(2, 13)
        d.profile = r.randint(0, 3)
        d.g0_bits_per_channel, d.g1_bits_per_channel = r.choice([(2, 4), (4, 4)])
        d.g0_channels, d.g1_channels = r.choice([(8, 12), (12, 20), (12, 10), (16, 12)])
        for i in range(levels):
            n0, n1 = r.randint(1, 300), r.randint(1, 300)
            b0 = np.frombuffer(bytes(r.randrange(256) for _ in range(n0)), np.uint8).copy()
            b1 = np.frombuffer(bytes(r.randrange(256) for _ in range(n1)), np.uint8).copy()
            self.keep += [b0, b1]
            d.g0[i] = b0.ctypes.data_as(C.POINTER(C.c_uint32))
            d.g1[i] = b1.ctypes.data_as(C.POINTER(C.c_uint32))
            d.g0_size[i], d.g1_size[i] = n0, n1
            d.g0_grid_dim[i], d.g1_grid_dim[i] = r.randint(1, 4096), r.randint(1, 2048)
        nd = r.randint(1, 12000)
        bd = np.frombuffer(bytes(r.randrange(256) for _ in range(nd)), np.uint8).copy()
        self.keep.append(bd)
        d.decoder, d.decoder_size = bd.ctypes.data, nd
        d.channel_count = r.randint(0, 16)
        for i in range(d.channel_count):
            d.channel_semantics[i] = r.randint(1, 11)
        vals = []
        for _ in range(4):
            kind = r.randrange(5)
            if kind == 0:
                v = struct.unpack("f", struct.pack("I", r.getrandbits(32) & 0x7F7FFFFF))[0]
            elif kind == 1:
                v = r.uniform(0, 10)
            elif kind == 2:
                v = r.uniform(0, 1e-3)
            elif kind == 3:
                v = float(r.randint(0, 10 ** 7))
            else:
                v = r.choice([0.0, 1.0, 1e-5, 123456789.0, 1e16, 1e-4, 0.1, 3.0])
            vals.append(v)
        d.caldata.max_abs_a1, d.caldata.max_abs_a2, d.caldata.s_a1, d.caldata.s_a2 = vals
        self.data = d


def corruptions(raw: bytes) -> dict[str, bytes]:
    """Malformed variants of a valid container, each hitting one of Load's checks
    (openntc_runtime.cpp:318-431)."""
    import json
    hdr = struct.unpack("4I", raw[:16])
    jlen = hdr[2]
    js = json.loads(raw[16:16 + jlen])
    blobs = raw[16 + jlen:]

    def rebuild(obj, h1=4, magic=0x43544E4F, blob_bytes=None):
        s = json.dumps(obj, separators=(",", ":")).encode()
        b = blobs if blob_bytes is None else blob_bytes
        return struct.pack("4I", magic, h1, len(s), len(b)) + s + b

    out = {
        "empty": b"",
        "short_header": raw[:10],
        "bad_magic": rebuild(js, magic=0x12345678),
        "bad_version": rebuild(js, h1=5),
        "bad_json": struct.pack("4I", hdr[0], 4, 5, 0) + b"{bad}",
    }
    for key in ("g0", "g1", "calibration", "dim", "mip_count", "level_count", "profile", "channel_semantics", "blobs"):
        o = dict(js)
        del o[key]
        out[f"missing_{key}"] = rebuild(o)
    o = json.loads(json.dumps(js))
    o["profile"] = "bpp_9_9"
    out["unknown_profile"] = rebuild(o)
    o = json.loads(json.dumps(js))
    o["channel_semantics"] = ["Albedo", "Bogus"]
    out["unknown_semantic"] = rebuild(o)
    o = json.loads(json.dumps(js))
    o["level_count"] = 7
    out["too_many_levels"] = rebuild(o)
    o = json.loads(json.dumps(js))
    o["mip_count"] = 0
    out["zero_mips"] = rebuild(o)
    o = json.loads(json.dumps(js))
    o["g0"]["grid_dims"] = o["g0"]["grid_dims"][:5]
    out["short_grid_dims"] = rebuild(o)
    o = json.loads(json.dumps(js))
    o["g1"]["bits"] = 4.5
    out["float_bits"] = rebuild(o)
    o = json.loads(json.dumps(js))
    o["blobs"] = o["blobs"][:-1]
    out["missing_blob"] = rebuild(o)
    o = json.loads(json.dumps(js))
    o["blobs"][0]["size"] = 10 ** 9
    out["blob_past_end"] = rebuild(o)
    o = json.loads(json.dumps(js))
    o["calibration"]["s_a1"] = "x"
    out["string_calibration"] = rebuild(o)
    o = json.loads(json.dumps(js))
    o["channel_semantics"] = ["Albedo"] * 17
    out["too_many_channels"] = rebuild(o)
    return out

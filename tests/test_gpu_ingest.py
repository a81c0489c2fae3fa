"""LoadManifest's ingest chain fused with packaging (one kernel per mip writes the source's mip
and its channels of the target package; upstream libopenntc.cpp:1296-1362 runs prepare, two
Lanczos passes per mip and a package pass).

The Lanczos reduction is applied per channel with the same taps, so channel k of the package at
mip m + 1 must equal the two-kernel reduction (ontc_debug_lanczos_down, itself pinned to
upstream's filter_lanczos) of channel k at mip m, bit for bit, for every mip of the chain.  Sizes
from 16 to 256 put whole CTA tiles, partial tiles and tiles wider than the mip in the chain, and
4 / 12 channels interleave one to four sources.  The chain and package at 1024^2 are also
compared with upstream itself in test_gpu_parity.py."""
import ctypes as C

import numpy as np
import pytest

import openntc_b200 as ont
from openntc_b200.synth import make_material
from tests import helpers as H

pytestmark = pytest.mark.gpu


def _down(lib, img):
    d, c = img.shape[0], img.shape[2]
    out = np.zeros((d // 2, d // 2, c), np.uint8)
    assert lib.ontc_debug_lanczos_down(np.ascontiguousarray(img).ctypes.data_as(C.c_void_p), d, c,
                                       out.ctypes.data_as(C.c_void_p)) == 0
    return out


@pytest.mark.parametrize("dim,channels,seed", [(16, 4, 31), (64, 12, 32), (256, 9, 33), (128, 6, 34)])
def test_fused_chain_matches_two_kernel_reduction(lib, tmp_path, dim, channels, seed):
    manifest = make_material(tmp_path, dim, seed=seed, channels=channels)
    ctx = ont.Context()
    assert ctx.init(ont.Profile.Bpp_1_0) == ont.Result.Success
    assert ctx.set_min_dimension(16) == ont.Result.Success
    assert ctx.load_manifest(manifest) == ont.Result.Success
    sh = H.shape(ctx)
    Cn = sh["C"]
    assert Cn == channels
    prev = None
    for m in range(sh["mips"]):
        d = sh["mip_dim"][m]
        pkg = H.package(ctx, m, d * d * Cn).reshape(d, d, Cn)
        if prev is not None:
            for k in range(Cn):
                want = _down(lib, prev[:, :, k:k + 1])[:, :, 0]
                assert np.array_equal(pkg[:, :, k], want), (dim, m, k)
        prev = pkg
    ctx.destroy()

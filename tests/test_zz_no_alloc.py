"""ontc_lanczos_down_noalloc: the mip reduction on caller-owned device buffers with no device
allocation (scratch in a fixed device array).  Compared, bit for bit, with the allocating
entry point ontc_debug_lanczos_down on the same images, over calls in a row that reuse the
scratch.  Named to run after every other test file; it also passes on its own."""
import ctypes as C

import numpy as np
import pytest

from openntc_b200 import _abi

pytestmark = pytest.mark.gpu

LIMIT = 2097152  # ONTC_NOALLOC_SCRATCH_FLOATS


def _image(dim, ch, seed):
    rng = np.random.default_rng(seed)
    base = rng.integers(0, 256, (dim, dim, ch), dtype=np.uint8)
    # smooth regions and hard edges both, so the taps' renormalisation at borders is exercised
    ramp = (np.arange(dim, dtype=np.uint32)[None, :, None] * 255 // max(1, dim - 1)).astype(np.uint8)
    return np.where(rng.random((dim, dim, 1)) < 0.5, base, np.broadcast_to(ramp, base.shape)).copy()


def _allocating(lib, img):
    dim, ch = img.shape[0], img.shape[2]
    out = np.zeros((dim // 2, dim // 2, ch), np.uint8)
    assert lib.ontc_debug_lanczos_down(img.ctypes.data_as(C.c_void_p), dim, ch, out.ctypes.data_as(C.c_void_p)) == 0
    return out


def _noalloc(lib, torch, img, stream):
    dim, ch = img.shape[0], img.shape[2]
    src = torch.from_numpy(img).cuda()
    dst = torch.full((dim // 2, dim // 2, ch), 7, dtype=torch.uint8, device="cuda")
    # src and dst were written on torch's current stream: the reduction's stream waits for them
    stream.wait_stream(torch.cuda.current_stream())
    r = lib.ontc_lanczos_down_noalloc(C.c_void_p(src.data_ptr()), dim, ch, C.c_void_p(dst.data_ptr()),
                                      C.c_void_p(stream.cuda_stream))
    assert r == 0, r
    stream.synchronize()
    return dst.cpu().numpy()


@pytest.fixture(scope="module")
def torch_cuda():
    torch = pytest.importorskip("torch")
    if not torch.cuda.is_available():
        pytest.skip("no CUDA device")
    return torch


def test_noalloc_matches_allocating_entry_point_on_calls_in_a_row(lib, torch_cuda):
    torch = torch_cuda
    stream = torch.cuda.Stream()
    # largest image first, then smaller ones: a later call reads only what it wrote itself
    cases = [(1024, 4, 1), (512, 3, 2), (256, 1, 3), (2048, 1, 4), (64, 2, 5), (2, 4, 6)]
    for dim, ch, seed in cases:
        img = _image(dim, ch, seed)
        want = _allocating(lib, img)
        assert dim * (dim // 2) * ch <= LIMIT
        got = _noalloc(lib, torch, img, stream)
        assert np.array_equal(got, want), (dim, ch)
    # the same image twice in a row on the default stream
    img = _image(128, 4, 9)
    want = _allocating(lib, img)
    for _ in range(2):
        assert np.array_equal(_noalloc(lib, torch, img, torch.cuda.default_stream()), want)


def test_noalloc_rejects_images_beyond_its_scratch(lib, torch_cuda):
    torch = torch_cuda
    src = torch.zeros(16, dtype=torch.uint8, device="cuda")
    dst = torch.zeros(16, dtype=torch.uint8, device="cuda")
    too_big = [(2048, 2), (4096, 1), (1448, 4)]
    for dim, ch in too_big:
        assert dim * (dim // 2) * ch > LIMIT
        r = lib.ontc_lanczos_down_noalloc(C.c_void_p(src.data_ptr()), dim, ch, C.c_void_p(dst.data_ptr()), None)
        assert r == 1, (dim, ch, r)  # ONTC_INVALID_DIMENSION, nothing enqueued
    for dim, ch in [(1, 1), (64, 0), (64, 5)]:
        assert lib.ontc_lanczos_down_noalloc(C.c_void_p(src.data_ptr()), dim, ch, C.c_void_p(dst.data_ptr()), None) == 1
    assert lib.ontc_lanczos_down_noalloc(None, 64, 1, C.c_void_p(dst.data_ptr()), None) == 1
    torch.cuda.synchronize()
    assert not dst.any()


def test_noalloc_calls_allocate_no_device_memory(lib, torch_cuda):
    """The property the entry point exists for: after a first call (which looks the scratch array
    up), further calls leave the device's free memory unchanged."""
    torch = torch_cuda
    img = _image(512, 4, 11)
    src = torch.from_numpy(img).cuda()
    dst = torch.zeros((256, 256, 4), dtype=torch.uint8, device="cuda")
    stream = torch.cuda.Stream()
    stream.wait_stream(torch.cuda.current_stream())

    def call():
        assert lib.ontc_lanczos_down_noalloc(C.c_void_p(src.data_ptr()), 512, 4, C.c_void_p(dst.data_ptr()),
                                             C.c_void_p(stream.cuda_stream)) == 0
        stream.synchronize()

    call()
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for _ in range(8):
        call()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0
    assert np.array_equal(dst.cpu().numpy(), _allocating(lib, img))

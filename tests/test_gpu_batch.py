"""ontc_train_batch: several contexts advanced together give the same training as separate
ontc_train calls: FP32 / BF16X3 contexts by interleaving their chunks on their own streams,
BF16 contexts in lock step with one shared tcgen05 tile launch per profile shape and step
(the SMs split among the materials by the tile autotuner's measured costs)."""
import numpy as np
import pytest

import openntc_b200 as ont
from tests import helpers as H

pytestmark = pytest.mark.gpu

# a mixed batch: channel counts, profiles and sizes differ per material
MIX = [(256, 4, ont.Profile.Bpp_0_2), (256, 6, ont.Profile.Bpp_0_5), (512, 9, ont.Profile.Bpp_1_0),
       (256, 12, ont.Profile.Bpp_2_25)]


def _contexts(materials, steps):
    return [H.new_context(p, materials(dim, 20 + i, ch), min_dim=16, grids=2, steps=steps,
                          precision=ont.Precision.FP32)
            for i, (dim, ch, p) in enumerate(MIX)]


def test_batch_matches_separate_training(materials):
    steps = 120  # the lock (step 114) and the completion fall inside the run
    solo = _contexts(materials, steps)
    for c in solo:
        p = c.train(70)
        assert p.result == 0 and p.batches_complete == 70
    batch = _contexts(materials, steps)
    r, prog = ont.train_batch(batch, 70)
    assert r == ont.Result.Success
    assert [p.batches_complete for p in prog] == [70] * len(MIX)
    # the rest in one more batch call: every context completes
    r, prog = ont.train_batch(batch, 1000)
    assert r == ont.Result.Success
    assert all(p.phase == ont.TrainPhase.TrainComplete and p.batches_complete == steps for p in prog)
    for c in solo:
        assert c.train_until_complete().phase == ont.TrainPhase.TrainComplete
    for a, b in zip(solo, batch):
        la, lb = np.array(a.step_losses(steps)), np.array(b.step_losses(steps))
        assert np.allclose(la, lb, rtol=1e-3, atol=0), np.abs(la - lb).max()
        assert abs(a.eval().psnr - b.eval().psnr) < 0.01
        ca, cb = a.get_compressed_data(), b.get_compressed_data()
        assert ca.decoder_size == cb.decoder_size and ca.level_count == cb.level_count


def test_batch_rejects_a_context_twice_and_reports_finished_ones(materials):
    ctxs = _contexts(materials, 30)[:2]
    r, _ = ont.train_batch([ctxs[0], ctxs[0]], 5)
    assert r == ont.Result.InvalidState
    assert ctxs[0].train_until_complete().phase == ont.TrainPhase.TrainComplete
    r, prog = ont.train_batch(ctxs, 10)  # one complete, one fresh
    assert r == ont.Result.Success
    assert prog[0].phase == ont.TrainPhase.TrainComplete and prog[0].batches_complete == 30
    assert prog[1].phase == ont.TrainPhase.TrainInProgress and prog[1].batches_complete == 10


# BF16 contexts share their tile launches: one tcgen05 launch per profile shape and step, the
# SMs split among that step's materials (three Bpp_1_0 materials share one launch here)
MIX_BF16 = [(256, 9, ont.Profile.Bpp_1_0), (512, 9, ont.Profile.Bpp_1_0), (256, 4, ont.Profile.Bpp_0_2),
            (256, 12, ont.Profile.Bpp_2_25), (512, 6, ont.Profile.Bpp_1_0)]


def _bf16_contexts(materials, steps):
    return [H.new_context(p, materials(dim, 40 + i, ch), min_dim=16, grids=2, steps=steps,
                          precision=ont.Precision.BF16)
            for i, (dim, ch, p) in enumerate(MIX_BF16)]


def _tile_launches(ctx):
    """Tile-kernel launches of the context so far (its kernel profile, ontc_kernel_times)."""
    from openntc_b200 import _abi
    kt = (_abi.KernelTime * _abi.KCLASS_COUNT)()
    assert ctx._lib.ontc_kernel_times(ctx.handle, kt, _abi.KCLASS_COUNT) == _abi.KCLASS_COUNT
    return kt[_abi.KCLASS_UNITS_BF16].launches


def test_bf16_batch_shares_tile_launches(materials):
    """The shared launches train every material as its own ontc_train does, within the run-to-run
    spread of the bf16 tile kernel (its decoder gradients are summed in arrival order): step
    losses within 2 %, final PSNR within 0.05 dB.  The kernel profile shows the sharing: a
    shared launch is one tile launch (of its first material) per profile shape and step."""
    steps = 120
    solo = _bf16_contexts(materials, steps)
    for c in solo:
        assert c.train(70).result == 0
        assert c._lib.ontc_profile_kernels(c.handle, 1) == 0
        assert c.train(1000).phase == ont.TrainPhase.TrainComplete
        assert _tile_launches(c) == steps - 70
    batch = _bf16_contexts(materials, steps)
    r, prog = ont.train_batch(batch, 70)  # also times the autotuner's trials
    assert r == ont.Result.Success and [p.batches_complete for p in prog] == [70] * len(MIX_BF16)
    for c in batch:
        assert c._lib.ontc_profile_kernels(c.handle, 1) == 0
    r, prog = ont.train_batch(batch, 1000)
    assert r == ont.Result.Success
    assert all(p.phase == ont.TrainPhase.TrainComplete and p.batches_complete == steps for p in prog)
    shapes = len({p for _, _, p in MIX_BF16})
    assert sum(_tile_launches(c) for c in batch) == (steps - 70) * shapes
    for a, b in zip(solo, batch):
        la, lb = np.array(a.step_losses(steps)), np.array(b.step_losses(steps))
        assert np.all(np.isfinite(lb))
        assert np.allclose(la, lb, rtol=2e-2, atol=0), np.abs(la / lb - 1).max()
        assert abs(a.eval().psnr - b.eval().psnr) < 0.05


def test_tile_autotuner_times_each_lod_once_and_caches(materials, tmp_path, monkeypatch):
    """ontc_train_batch splits a shared launch's SMs by the measured cost of a unit round at
    each material's lod: timed once per lod (one warm-up and three timed trial launches), then
    read back from the cache file by any context of the same shape and sizes."""
    import ctypes as C
    cache = tmp_path / "tile_costs.txt"
    monkeypatch.setenv("ONTC_TUNE_CACHE", str(cache))
    manifest = materials(512, 50, 9)

    def costs(ctx):
        n = H.shape(ctx)["mips"]
        buf = (C.c_float * n)()
        before = ctx.kernel_launches()
        assert ctx._lib.ontc_debug_tile_costs(ctx.handle, buf, n) == 0
        return list(buf), ctx.kernel_launches() - before

    a = H.new_context(ont.Profile.Bpp_1_0, manifest, min_dim=16, grids=2, steps=20, precision=ont.Precision.BF16)
    first, launched = costs(a)
    assert all(c > 0 for c in first) and launched == 4 * len(first)
    assert len(cache.read_text().splitlines()) == len(first)
    again, launched = costs(a)
    assert again == first and launched == 0
    b = H.new_context(ont.Profile.Bpp_1_0, manifest, min_dim=16, grids=2, steps=20, precision=ont.Precision.BF16)
    cached, launched = costs(b)
    assert launched == 0 and np.allclose(cached, first, rtol=1e-3, atol=1e-4)
    # the trials leave the training state alone: training after them still completes and learns
    p = a.train_until_complete()
    assert p.phase == ont.TrainPhase.TrainComplete and np.isfinite(a.eval().psnr)

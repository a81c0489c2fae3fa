"""ontc_train_batch: several contexts advanced together (their chunks interleaved so their
kernels overlap on the GPU) give the same training as separate ontc_train calls."""
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

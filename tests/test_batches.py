"""The frame's tile-batch schedule (TileRegion and TraceProgress of the reference,
crates/gravlume-render/src/trace.rs:799-857 and renderer/frame.rs:326-420), host logic only:
the reference's own tests restated (frame.rs:499-580), plus the schedule's budget arithmetic."""

import numpy as np
import pytest

from gravlume_b200.batches import (MAXIMUM_BATCH_MS, TARGET_BATCH_MS, TileRegion, TraceProgress, tile_grid)


def _run(width, height, mdd, ms=TARGET_BATCH_MS):
    progress = TraceProgress(width, height, mdd)
    gx, gy = tile_grid(width, height)
    covered = np.zeros((gy, gx), dtype=bool)
    batches = []
    while (batch := progress.next_batch()) is not None:
        (ox, oy), (wx, wy) = batch.origin, batch.workgroups
        assert wx <= mdd and wy <= mdd
        assert ox + wx <= gx and oy + wy <= gy
        assert not covered[oy:oy + wy, ox:ox + wx].any(), "a tile was repeated"
        covered[oy:oy + wy, ox:ox + wx] = True
        progress.submitted(batch)
        assert progress.next_batch() is None, "one batch stays in flight"
        progress.completed(ms(batch) if callable(ms) else ms)
        batches.append(batch)
    assert covered.all()
    assert progress.next_batch() is None and progress.done
    return batches


def test_schedule_covers_native_extents_once_with_bounded_batches():
    """trace_progress_covers_native_extents_once_with_bounded_batches (frame.rs:499-532), 128
    seeded cases of width 1..3840, height 1..2160 and dispatch limit 1..512."""
    rng = np.random.default_rng(128)
    for _ in range(128):
        _run(int(rng.integers(1, 3841)), int(rng.integers(1, 2161)), int(rng.integers(1, 513)))


def test_only_the_last_batch_finishes_the_frame():
    """publication_gate_requires_the_complete_current_generation (frame.rs:535-558), the
    4097x9 extent at the default dispatch limit."""
    progress = TraceProgress(4097, 9, 65535)
    covered = 0
    while (batch := progress.next_batch()) is not None:
        progress.submitted(batch)
        covered += len(batch)
        assert batch.finishes(4097, 9) == (covered == progress.total_tiles)
        progress.completed(TARGET_BATCH_MS)


def test_batches_are_row_runs_or_whole_row_blocks():
    for b in _run(1000, 300, 65535, ms=lambda b: 10.0):
        gx, _ = tile_grid(1000, 300)
        assert b.workgroups[1] == 1 or (b.origin[0] == 0 and b.workgroups[0] == gx)


def test_budget_rescales_towards_the_target():
    p = TraceProgress(3840, 2160)
    b = p.next_batch()
    # a budget of 512 tiles covers one whole row of the 480-tile-wide grid
    assert b.origin == (0, 0) and b.workgroups == (480, 1)
    p.submitted(b)
    p.completed(TARGET_BATCH_MS / 4)  # fast: grows by the maximum factor 1.5
    assert p.tiles_per_batch == 720
    b = p.next_batch()
    p.submitted(b)
    p.completed(TARGET_BATCH_MS)  # on target: unchanged
    assert p.tiles_per_batch == len(b)
    b = p.next_batch()
    p.submitted(b)
    p.completed(MAXIMUM_BATCH_MS + 1)  # over the ceiling: halved
    assert p.tiles_per_batch == round(len(b) * 0.5)


def test_region_rectangles_clip_to_the_view():
    assert TileRegion.all(1001, 17).workgroups == (126, 3)
    assert TileRegion.all(1001, 17).pixel_rect(1001, 17) == (0, 0, 1001, 17)
    assert TileRegion((125, 2), (1, 1)).pixel_rect(1001, 17) == (1000, 16, 1001, 17)
    assert TileRegion.containing_pixel(17, 9) == TileRegion((2, 1), (1, 1))
    with pytest.raises(ValueError):
        TileRegion((0, 0), (0, 1))

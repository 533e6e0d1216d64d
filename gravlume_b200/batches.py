"""Tile batches of a frame, in the reference's terms: TileRegion (crates/gravlume-render/src/
trace.rs:799-857) and the progressive batch schedule of TraceProgress (crates/gravlume-render/src/
renderer/frame.rs:326-420), which the renderer uses to keep each trace submission under a time
budget (its watchdog control).

A region is a block of 8x8-pixel tiles: its origin (column, row) and its extent (columns, rows).
glc_trace takes it in glc_camera.tile_origin / tile_count, traces only those pixels and writes
them in the whole view's result layout, so a frame traced batch by batch equals the frame traced
at once. The batch arithmetic is the reference's, restated: a batch is either a run of tiles
along one tile row, or whole tile rows when the budget covers at least one row from column 0;
after each batch the budget is rescaled towards a 32 ms target (by 0.5 to 1.5, and by 0.5 when a
batch took more than 50 ms)."""

from __future__ import annotations

from dataclasses import dataclass

TRACE_WORKGROUP_AXIS = 8  # pixels per tile side (trace.rs:20)
INITIAL_TILES_PER_BATCH = 512
TARGET_BATCH_MS = 32.0
MAXIMUM_BATCH_MS = 50.0
MAXIMUM_BATCH_SCALE = 1.5
MINIMUM_BATCH_SCALE = 0.5


def tile_grid(width: int, height: int) -> tuple[int, int]:
    """Tiles (columns, rows) covering a width x height view (trace.rs:851-856)."""
    return (-(-width // TRACE_WORKGROUP_AXIS), -(-height // TRACE_WORKGROUP_AXIS))


@dataclass(frozen=True)
class TileRegion:
    origin: tuple[int, int]
    workgroups: tuple[int, int]

    def __post_init__(self):
        if self.workgroups[0] <= 0 or self.workgroups[1] <= 0:
            raise ValueError("a tile region covers at least one tile")

    @staticmethod
    def all(width: int, height: int) -> "TileRegion":
        return TileRegion((0, 0), tile_grid(width, height))

    @staticmethod
    def containing_pixel(px: int, py: int) -> "TileRegion":
        return TileRegion((px // TRACE_WORKGROUP_AXIS, py // TRACE_WORKGROUP_AXIS), (1, 1))

    def __len__(self) -> int:
        return self.workgroups[0] * self.workgroups[1]

    def finishes(self, width: int, height: int) -> bool:
        """True when this batch ends the frame's row-major tile order (trace.rs:842-849)."""
        gx, gy = tile_grid(width, height)
        row_contiguous = self.workgroups[1] == 1 or (self.origin[0] == 0 and self.workgroups[0] == gx)
        return (row_contiguous and self.origin[0] + self.workgroups[0] == gx
                and self.origin[1] + self.workgroups[1] == gy)

    def pixel_rect(self, width: int, height: int) -> tuple[int, int, int, int]:
        """(x0, y0, x1, y1): the pixels the region traces, clipped to the view."""
        a = TRACE_WORKGROUP_AXIS
        return (self.origin[0] * a, self.origin[1] * a, min(width, (self.origin[0] + self.workgroups[0]) * a),
                min(height, (self.origin[1] + self.workgroups[1]) * a))


class TraceProgress:
    """The batch schedule of one frame: next_batch, submitted, completed (frame.rs:326-420)."""

    def __init__(self, width: int, height: int, maximum_dispatch_dimension: int = 65535,
                 tiles_per_batch: int | None = None):
        if maximum_dispatch_dimension <= 0:
            raise ValueError("maximum_dispatch_dimension must be positive")
        self.grid = tile_grid(width, height)
        self.total_tiles = self.grid[0] * self.grid[1]
        gx, gy = self.grid
        mdd = maximum_dispatch_dimension
        self.maximum_batch_tiles = mdd if gx > mdd else gx * (gy if gy < mdd else mdd)
        self.maximum_dispatch_dimension = mdd
        start = INITIAL_TILES_PER_BATCH if tiles_per_batch is None else int(tiles_per_batch)
        self.tiles_per_batch = min(start, self.maximum_batch_tiles)
        self.next_tile = 0
        self.in_flight: TileRegion | None = None
        self.completed_batches = 0
        self.total_compute_ms = 0.0
        self.maximum_batch_ms = 0.0

    def next_batch(self) -> TileRegion | None:
        if self.in_flight is not None or self.next_tile == self.total_tiles:
            return None
        gx, gy = self.grid
        tile_x, tile_y = self.next_tile % gx, self.next_tile // gx
        budget = min(self.tiles_per_batch, self.total_tiles - self.next_tile)
        wx = min(budget, gx - tile_x, self.maximum_dispatch_dimension)
        if tile_x == 0 and wx == gx and budget >= gx:
            wy = min(budget // gx, gy - tile_y, self.maximum_dispatch_dimension)
        else:
            wy = 1
        return TileRegion((tile_x, tile_y), (wx, wy))

    def submitted(self, batch: TileRegion) -> None:
        assert batch.origin[1] * self.grid[0] + batch.origin[0] == self.next_tile
        assert self.in_flight is None
        self.next_tile += len(batch)
        self.in_flight = batch

    def completed(self, compute_ms: float) -> None:
        batch, self.in_flight = self.in_flight, None
        if batch is None:
            return
        self.completed_batches += 1
        finite = compute_ms == compute_ms and compute_ms not in (float("inf"), float("-inf"))
        if finite:
            self.total_compute_ms += compute_ms
            self.maximum_batch_ms = max(self.maximum_batch_ms, compute_ms)
        if self.next_tile == self.total_tiles or not finite or compute_ms <= 0.0:
            return
        if compute_ms > MAXIMUM_BATCH_MS:
            scale = MINIMUM_BATCH_SCALE
        else:
            scale = min(max(TARGET_BATCH_MS / compute_ms, MINIMUM_BATCH_SCALE), MAXIMUM_BATCH_SCALE)
        scaled = min(max(round(len(batch) * scale), 1.0), float(min(self.total_tiles, self.maximum_batch_tiles)))
        self.tiles_per_batch = int(scaled)

    @property
    def done(self) -> bool:
        return self.next_tile == self.total_tiles and self.in_flight is None

"""The reference's CPU triangleBudget controller, restated for the host mirror.

VirtualGeometry.ts keeps the drawn triangle count near `triangleBudget` by steering `errorThreshold` from stats
readbacks (adaptThreshold, :549-567) and gliding toward the chosen value a few percent per frame (stepThreshold,
:575-588): it acts only after two readbacks in a row outside a +-15% band, aims at t * sqrt(drawn / budget) clamped to
`thresholdRange`, never refines past the threshold that would fill about 82% of the fullest draw buffer
(refineThreshold, :60), drops a refining target once the buffers are 75% full, moves at most x1.03 (coarser) or
/1.01 (finer) per frame, and lets a threshold set by the user win over a glide in progress. Readbacks happen every
`statsInterval` frames, every other frame while a glide is under way (:494-506).

The engine also offers the device search (`vgc_view.triangle_budget`): the threshold of the frame's own cut is
picked on the GPU from a log-error histogram, with no readback and no lag. `GlideController` is the reference's
behaviour for callers that want it (`VirtualGeometry(budget_mode="glide")`).
"""
from __future__ import annotations

import math

THRESHOLD_RATE_UP = 1.03    # VirtualGeometry.ts:21
THRESHOLD_RATE_DOWN = 1.01  # VirtualGeometry.ts:22


def refine_threshold(threshold: float, use: float) -> float:
    """Threshold at which a cut that filled `use` of its draw buffers at `threshold` fills about 82% (:60)."""
    return threshold * math.pow(use / 0.82, 0.25)


class GlideController:
    """State of the reference's budget controller for one VirtualGeometry (one camera)."""

    def __init__(self, error_threshold: float = 1.0, triangle_budget: float = 0.0,
                 threshold_range: tuple = (0.5, 3.0), stats_interval: int = 10):
        self.error_threshold = float(error_threshold)
        self.triangle_budget = float(triangle_budget)
        self.threshold_range = tuple(threshold_range)
        self.stats_interval = int(stats_interval)
        self.frame_count = 0
        self.out_of_band = 0
        self.target: float | None = None
        self.written = math.nan
        self.stats_threshold = 1.0

    def step(self) -> float:
        """Start of a frame (stepThreshold): moves the threshold toward the target; returns this frame's value."""
        t = self.error_threshold
        if t != self.written and not math.isnan(self.written):
            self.target = None  # set by the user: their value wins over a glide in progress
        if self.target is not None:
            target = self.target
            nxt = min(target, t * THRESHOLD_RATE_UP) if target > t else max(target, t / THRESHOLD_RATE_DOWN)
            self.error_threshold = nxt
            if nxt == target:
                self.target = None
        self.written = self.error_threshold
        return self.error_threshold

    def end_frame(self) -> bool:
        """End of a frame's update: counts it; True when this frame's stats should be read back (the caller then
        passes them to `adapt`)."""
        self.frame_count += 1
        interval = min(2, self.stats_interval) if self.target is not None else self.stats_interval
        if self.frame_count % interval == 0:
            self.stats_threshold = self.error_threshold
            return True
        return False

    def adapt(self, drawn_triangles: float, capacity_use: float) -> None:
        """A stats readback (adaptThreshold): picks the threshold to glide toward."""
        if self.triangle_budget <= 0:
            return
        t = self.stats_threshold
        now = self.error_threshold
        if self.target is not None and self.target < now and capacity_use >= 0.75:
            self.target = None  # refining, and the buffers are filling up: stop where we are
        if drawn_triangles <= 0:
            return
        ratio = drawn_triangles / self.triangle_budget
        if abs(ratio - 1) < 0.15:  # act only on a lasting difference
            self.out_of_band = 0
            return
        self.out_of_band += 1
        if self.out_of_band < 2:
            return
        lo, hi = self.threshold_range
        nxt = min(hi, max(lo, t * math.sqrt(ratio)))
        if nxt < t:  # refining multiplies the drawn triangles by about (t / next)^2: not into a full buffer
            nxt = max(nxt, refine_threshold(t, capacity_use))
        self.target = None if nxt == self.error_threshold else nxt


def stats_drawn_and_use(stats: dict, max_triangles: int, max_shadow_triangles: int, max_meshlets: int) -> tuple:
    """drawnTriangles and capacityUse of one readback (VirtualGeometry.readStats, :605-632) from vgc_stats."""
    req = [stats["requested_indices"][0] / 3.0, stats["requested_indices"][1] / 3.0]
    drawn = min(req[0], max_triangles)
    use = max(req[0] / max_triangles, stats["selected"][0] / max_meshlets,
              req[1] / max(1, max_shadow_triangles), stats["selected"][1] / max_meshlets)
    return drawn, use

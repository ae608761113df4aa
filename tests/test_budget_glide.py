"""The reference's CPU triangleBudget controller (VirtualGeometry.ts:549-588) as restated in vgcut.budget: each rule
on its own, then the closed loop on a model scene whose drawn triangles fall as 1 / threshold^2."""
import math

import pytest

from vgcut.budget import GlideController, refine_threshold, THRESHOLD_RATE_DOWN, THRESHOLD_RATE_UP


def readback(g, drawn, use=0.1):
    """One frame that reads stats: step, end of frame (must be a readback frame), adapt."""
    g.step()
    while not g.end_frame():
        g.step()
    g.adapt(drawn, use)


def test_deadband_and_two_readbacks():
    g = GlideController(1.0, 1000.0, (0.5, 3.0), stats_interval=1)
    readback(g, 1140.0)  # ratio 1.14: inside the +-15% band
    assert g.target is None and g.out_of_band == 0
    readback(g, 2000.0)  # out of band once: no action yet
    assert g.target is None and g.out_of_band == 1
    readback(g, 2000.0)  # twice in a row: aim at t * sqrt(2)
    assert g.target == pytest.approx(math.sqrt(2.0))
    readback(g, 1000.0)  # back in band: the counter resets (the glide continues)
    assert g.out_of_band == 0


def test_target_clamped_to_range():
    g = GlideController(2.0, 100.0, (0.5, 3.0), stats_interval=1)
    readback(g, 10_000.0)
    readback(g, 10_000.0)
    assert g.target == 3.0  # 2 * sqrt(100) clamped to the range's top


def test_glide_rates():
    g = GlideController(1.0, 1.0)
    g.target = 1.1
    assert g.step() == pytest.approx(THRESHOLD_RATE_UP)
    assert g.step() == pytest.approx(THRESHOLD_RATE_UP ** 2)
    assert g.step() == pytest.approx(THRESHOLD_RATE_UP ** 3)
    assert g.step() == 1.1 and g.target is None  # reached: the glide ends
    g.target = 1.0
    assert g.step() == pytest.approx(1.1 / THRESHOLD_RATE_DOWN)


def test_refining_stops_short_of_a_full_buffer():
    g = GlideController(2.0, 1000.0, (0.5, 3.0), stats_interval=1)
    readback(g, 250.0, use=0.7)
    readback(g, 250.0, use=0.7)
    # t * sqrt(0.25) = 1.0 would quadruple the triangles; refineThreshold(2, 0.7) = 2 * (0.7 / 0.82)^0.25 stops earlier
    assert g.target == pytest.approx(refine_threshold(2.0, 0.7))
    assert g.target > 1.0
    # a refining glide is dropped once the buffers are 75% full (here the count is back in band: no new target) ...
    g.step()
    g.adapt(1000.0, 0.8)
    assert g.target is None
    # ... and a still-low count needs two readbacks again (the in-band one reset the count), then aims capped by
    # refineThreshold at the new use
    g.stats_threshold = 2.0
    g.adapt(250.0, 0.8)
    assert g.target is None
    g.adapt(250.0, 0.8)
    assert g.target == pytest.approx(refine_threshold(2.0, 0.8))


def test_user_value_wins():
    g = GlideController(1.0, 1.0)
    g.target = 2.0
    g.step()
    g.error_threshold = 0.7  # set by the user between frames
    assert g.step() == 0.7 and g.target is None


def test_stats_interval_faster_while_gliding():
    g = GlideController(1.0, 1.0, stats_interval=10)
    frames = [i for i in range(1, 31) if (g.step(), g.end_frame())[1]]
    assert frames == [10, 20, 30]
    g.target = 5.0
    frames = [i for i in range(1, 7) if (g.step(), g.end_frame())[1]]
    assert frames == [2, 4, 6]  # frame_count 32, 34, 36: every other frame


def test_closed_loop_converges_to_the_budget():
    budget = 1_000_000.0
    k = budget * 2.0 ** 2  # drawn(t) = k / t^2: the budget is met at t = 2
    g = GlideController(1.0, budget, (0.5, 3.0), stats_interval=10)
    history = []
    for frame in range(600):
        t = g.step()
        drawn = k / t ** 2
        history.append(t)
        if g.end_frame():
            g.adapt(drawn, drawn / 20e6)
    final = k / history[-1] ** 2 / budget
    assert abs(final - 1) < 0.15
    # it got there by gliding: no frame changed the threshold by more than the rates allow
    for a, b in zip(history, history[1:]):
        assert b <= a * THRESHOLD_RATE_UP + 1e-12 and b >= a / THRESHOLD_RATE_DOWN - 1e-12

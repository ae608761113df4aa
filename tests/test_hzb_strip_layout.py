"""The HZB strip stream's layout (k_hzb_stream in csrc/vgcut_kernels.cu) restated on the CPU, against the oracle's max
reduction (OcclusionCulling.ts:320-350): 128 x 32 strips of mip 0; warp w of a block covers the 32 x 16 pixels at
(32 (w & 3), 16 (w >> 2)) of the strip, lane l the 4 x 4 patch at (4 (l & 7), 4 (l >> 3)) of those; levels 1-2 per
lane, level 3 over the lanes l ^ 1 and l ^ 8, level 4 over l ^ 2 and l ^ 16. A strip comes either from a bulk-tensor
copy (zeros past the image's edge, read back with indices clamped to the image) or from plain loads clamped to the
image. Every texel of levels 1-4 must be written and equal the oracle's, at sizes with partial strips on both edges
and images smaller than a strip."""
import numpy as np
import pytest

import oracle as O

SW, SH = 128, 32


def strip_levels(img: np.ndarray, tma: bool) -> tuple[np.ndarray, np.ndarray]:
    mips, levels, off, w, h = O.hzb_build(img)
    out = np.full(len(mips), np.nan, np.float32)
    H0, W0 = img.shape
    lane = np.arange(32)
    for oy in range(0, H0, SH):
        for ox in range(0, W0, SW):
            stage = np.zeros((SH, SW), np.float32)
            hh, ww = min(SH, H0 - oy), min(SW, W0 - ox)
            stage[:hh, :ww] = img[oy:oy + hh, ox:ox + ww]
            for warp in range(8):
                gx = ox + 32 * (warp & 3) + 4 * (lane & 7)  # per lane
                gy = oy + 16 * (warp >> 2) + 4 * (lane >> 3)
                r = np.arange(4)
                ys = np.minimum(gy[:, None] + r[None, :], H0 - 1)  # lane x row
                xs = np.minimum(gx[:, None] + r[None, :], W0 - 1)  # lane x column
                if tma:
                    assert (ys - oy).min() >= 0 and (ys - oy).max() < SH and (xs - ox).max() < SW
                    v = stage[(ys - oy)[:, :, None], (xs - ox)[:, None, :]]
                else:
                    v = img[ys[:, :, None], xs[:, None, :]]
                a = v.reshape(32, 2, 2, 2, 2).max(axis=(2, 4))  # lane, i, j: level 1
                b = a.max(axis=(1, 2))

                def store(level, x, y, val, mask):
                    if level >= levels:
                        return
                    ok = mask & (x < w[level]) & (y < h[level])
                    out[off[level] + y[ok] * w[level] + x[ok]] = val[ok]

                for i in range(2):
                    for j in range(2):
                        store(1, gx // 2 + j, gy // 2 + i, a[:, i, j], np.ones(32, bool))
                store(2, gx // 4, gy // 4, b, np.ones(32, bool))
                m3 = np.maximum(b, b[lane ^ 1])
                m3 = np.maximum(m3, m3[lane ^ 8])
                store(3, gx // 8, gy // 8, m3, (lane & 9) == 0)
                m4 = np.maximum(m3, m3[lane ^ 2])
                m4 = np.maximum(m4, m4[lane ^ 16])
                store(4, gx // 16, gy // 16, m4, (lane & 27) == 0)
    top = off[min(levels, 5)] if levels > 5 else len(mips)
    lo = off[1] if levels > 1 else len(mips)
    return out[lo:top], mips[lo:top]


@pytest.mark.parametrize("shape", [(77, 132), (33, 128), (130, 256), (300, 1004), (32, 132), (40, 36), (1, 4), (9, 1),
                                   (67, 129)])
def test_strip_layout_reproduces_the_mip_chain(shape):
    img = np.random.default_rng(shape[0] * 131 + shape[1]).random(shape, dtype=np.float32)
    for tma in (True, False):
        got, want = strip_levels(img, tma)
        assert not np.isnan(got).any(), "a texel of levels 1-4 is not written"
        assert np.array_equal(got, want)

"""The seeded Delaunay mesh of the unit square that stands for the 200k-triangle
configuration: minimum angle, orientation, size, determinism and the reference's
segment/triangle conventions (tri_mesh/setup.cpp:76-145)."""
import numpy as np

import hpb


def test_delaunay_square_quality_and_conventions():
    m = hpb.delaunay_square(64, seed=11)
    assert m.min_angle >= 20.0
    assert np.all(m.area2() > 0)
    assert abs(m.ntri - 2 * 64 * 64) < 0.05 * 2 * 64 * 64
    assert abs(np.sum(m.area2()) / 2 - 1.0) < 1e-12  # the triangles tile the unit square
    # seg j of a triangle is opposite pnt j; sgn = +1 when the segment runs CCW for it
    for t in range(0, m.ntri, 97):
        for j in range(3):
            s = m.tri_seg[t, j]
            a, b = m.tri_pnt[t, (j + 1) % 3], m.tri_pnt[t, (j + 2) % 3]
            if m.tri_sgn[t, j] > 0:
                assert (m.seg_pnt[s, 0], m.seg_pnt[s, 1]) == (a, b)
            else:
                assert (m.seg_pnt[s, 0], m.seg_pnt[s, 1]) == (b, a)
    bs = m.boundary_segments()
    mid = 0.5 * (m.pnts[m.seg_pnt[bs, 0]] + m.pnts[m.seg_pnt[bs, 1]])
    on = (np.abs(mid[:, 0]) < 1e-12) | (np.abs(mid[:, 0] - 1) < 1e-12) | (np.abs(mid[:, 1]) < 1e-12) | \
         (np.abs(mid[:, 1] - 1) < 1e-12)
    assert np.all(on)


def test_delaunay_square_is_seeded():
    a = hpb.delaunay_square(16, seed=5)
    b = hpb.delaunay_square(16, seed=5)
    c = hpb.delaunay_square(16, seed=6)
    assert np.array_equal(a.pnts, b.pnts) and np.array_equal(a.tri_pnt, b.tri_pnt)
    assert not np.array_equal(a.pnts, c.pnts)

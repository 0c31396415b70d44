"""h-level transfer weights (tri_mesh::mgconnect, tri_mesh/connect.cpp:49-86, with the
boundary re-connection of edge_bdry::mgconnect, tri_mesh/tri_boundary.cpp:164-201):
interior points take their containing triangle, boundary points the nearest boundary
side of the other mesh, so boundary values move between levels through boundary
values only."""
import numpy as np

import hpb
from hpb import multigrid as MG


def boundary_points(m):
    return np.unique(m.seg_pnt[m.boundary_segments()].ravel())


def check_boundary_weights(src, tgt, t, w):
    assert np.all(w >= -1e-12) and np.allclose(w.sum(1), 1.0, atol=1e-14)
    onb = np.zeros(tgt.npnt, bool)
    onb[boundary_points(tgt)] = True
    bp = boundary_points(src)
    used = tgt.tri_pnt[t[bp]]
    # weight only on the two end points of one boundary side of tgt
    assert np.all((w[bp] == 0.0) | onb[used])
    assert np.all(np.sum(w[bp] > 0.0, axis=1) <= 2)
    interp = np.einsum("kj,kjd->kd", w[bp], tgt.pnts[used])
    return bp, interp


def test_curved_hole_boundary_points_use_coarse_boundary_sides():
    f = hpb.channel_hole(L=4.0, H=2.0, cx=1.0, cy=1.0, r=0.25, hmin=0.04, hmax=0.15, grade=0.1)
    c = hpb.channel_hole(L=4.0, H=2.0, cx=1.0, cy=1.0, r=0.25, hmin=0.08, hmax=0.3, grade=0.2)
    cx, cy, r = f.hole
    for src, tgt in ((f, c), (c, f)):
        t0, w0 = MG.locate(tgt, src.pnts)
        t, w = MG.connect(src, tgt)
        bp, interp = check_boundary_weights(src, tgt, t, w)
        x = src.pnts[bp]
        hole = np.abs(np.hypot(x[:, 0] - cx, x[:, 1] - cy) - r) < 1e-9
        # hole points map to a chord of tgt's hole polygon: within its sagitta of the circle
        h = np.max(np.linalg.norm(tgt.pnts[tgt.seg_pnt[tgt.boundary_segments(), 1]] -
                                  tgt.pnts[tgt.seg_pnt[tgt.boundary_segments(), 0]], axis=1))
        rr = np.hypot(interp[hole, 0] - cx, interp[hole, 1] - cy)
        assert np.all(rr <= r + 1e-12) and np.all(rr >= r - h * h / (8 * r) - 1e-9)
        # straight walls: the point itself
        assert np.max(np.abs(interp[~hole] - x[~hole])) < 1e-12
        # containing-triangle weights of hole points reach an interior vertex (the reason
        # for the re-connection); the interior points keep them
        onb = np.zeros(tgt.npnt, bool)
        onb[boundary_points(tgt)] = True
        hp = bp[hole]
        assert np.any((w0[hp] > 1e-12) & ~onb[tgt.tri_pnt[t0[hp]]])
        inner = np.setdiff1d(np.arange(src.npnt), bp)
        assert np.array_equal(t[inner], t0[inner]) and np.array_equal(w[inner], w0[inner])


def test_nested_square_meshes_unchanged():
    f, c = hpb.square_mesh(8), hpb.square_mesh(4)
    for src, tgt in ((f, c), (c, f)):
        t0, w0 = MG.locate(tgt, src.pnts)
        t, w = MG.connect(src, tgt)
        bp, interp = check_boundary_weights(src, tgt, t, w)
        assert np.max(np.abs(interp - src.pnts[bp])) < 1e-13
        a = np.einsum("kj,kjd->kd", w0, tgt.pnts[tgt.tri_pnt[t0]])
        b = np.einsum("kj,kjd->kd", w, tgt.pnts[tgt.tri_pnt[t]])
        assert np.max(np.abs(a - b)) < 1e-13
